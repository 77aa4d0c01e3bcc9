"""Build recipe for oracle/_ref: the reference's own code, compiled on the host.

Test infrastructure only.  Compiles, from the files where they lie in the
reference tree (the first argument; else FORNOS_REF_ROOT; else a checkout
named `reference` beside this repository):

  * Src/bvh.cpp, Src/compute.cpp          verbatim, with a force-included shim
                                           (ref_shim.h) for the MSVC-only
                                           std::sqrtf-style names;
  * Src/meshmapping.cpp                    #included by ref_host_driver.cpp to
                                           reach fillMeshData (anonymous namespace);
  * Src/mesh.cpp lines 38-41 and 619-768   the Vector3 ordering and the normal /
                                           tangent generators;
  * Src/mesh.cpp lines 1-37 and 42-617,    the OBJ / PLY loaders, with two
    3rdParty/tinyply/tinyply.cpp           MSVC-only constructs spelled for g++
                                           (std::find_if over the overloaded
                                           std::isspace takes ::isspace, and a
                                           lambda bound to `auto &` is bound to
                                           `auto`); nothing else changes;
  * 3rdParty/glad/glad.c                   GL entry-point table the above refer
                                           to (never called: no GL context);
  * Src/image.cpp, 3rdParty/tinyexr/tinyexr.cc
                                           the image export (PNG / TGA through
                                           stb_image_write, EXR through tinyexr),
                                           with its exportNormalImage renamed
                                           ref_exportNormalImage: CompressedMapUV's
                                           constructor calls that name for a
                                           debug file (Src/compute.cpp:413-415),
                                           which the driver keeps a no-op;
  * Shaders/*.comp                         rewritten on the fly to C++ (buffer and
                                           uniform declarations become thread-
                                           local globals,
                                           in/out parameters become references,
                                           float literals get an f suffix) and
                                           compiled against ref_glsl.h.

Sources are piped to the compiler; nothing from the reference tree is written
into this repository.  Output: oracle/_ref/libfornos_ref.so (+ objects in
oracle/_ref/obj).  Exit status 0 on success; prints the reason and exits 1 when
the reference tree is absent.
"""
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
OBJ = os.path.join(OUT, "obj")
REPO = os.path.dirname(HERE)
REF = (sys.argv[1] if len(sys.argv) > 1 else
       os.environ.get("FORNOS_REF_ROOT", os.path.join(os.path.dirname(REPO), "reference")))

CXX = ["g++", "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-w"]

SHADERS = [
    "meshmapping", "meshmapping_nobackfaces", "ao_step0", "ao_step1", "ao_step2",
    "bentnormals_step1", "bentnormals_step2", "thick_step1", "thick_step2",
    "heights", "positions", "normals", "tangentspace",
]

FLOAT_LIT = re.compile(
    r"(?<![\w.])(\d+\.\d*(?:[eE][+-]?\d+)?|\.\d+(?:[eE][+-]?\d+)?|\d+[eE][+-]?\d+)(?![\w.])")


def glsl_to_cpp(src, name):
    """Rewrites one compute shader into a C++ namespace `sh_<name>`."""
    out = []
    defines = []
    shadow_depth = None  # brace depth at which a renamed barycentric local lives
    depth = 0
    for line in src.splitlines():
        s = line.strip()
        if s.startswith("#version") or s.startswith("#extension"):
            continue
        if re.match(r"layout\s*\(\s*local_size_x", s):
            continue
        m = re.match(r"#define\s+(\w+)", s)
        if m:
            defines.append(m.group(1))
        m = re.match(r"layout\s*\(\s*location\s*=\s*\d+\s*\)\s*uniform\s+(\w+)\s+(\w+)\s*;", s)
        if m:
            out.append("static thread_local %s %s;" % (m.group(1), m.group(2)))
            continue
        m = re.match(r"layout\s*\(\s*std430\s*,\s*binding\s*=\s*\d+\s*\)\s*(?:readonly\s+|writeonly\s+)?"
                     r"buffer\s+\w+\s*\{\s*(\w+)\s+(\w+)\s*(\[\])?\s*;\s*\}\s*;", s)
        if m:
            star = "*" if m.group(3) else ""
            out.append("static thread_local %s%s %s;" % (m.group(1), star, m.group(2)))
            continue
        line = re.sub(r"\bin\s+out\s+(\w+)\s+(\w+)", r"\1& \2", line)
        line = re.sub(r"\bout\s+(\w+)\s+(\w+)", r"\1& \2", line)
        line = FLOAT_LIT.sub(lambda mm: mm.group(1) + "f", line)
        line = line.replace(".yzw", ".yzw()")
        # GLSL scopes a declared name after its initializer; C++ before it.
        # `vec3 b = barycentric(p, a, b, c);` therefore gets a distinct name.
        if re.search(r"\bvec3\s+b\s*=\s*barycentric\(", line):
            line = re.sub(r"\bvec3\s+b\s*=", "vec3 bary_ =", line)
            shadow_depth = depth
        elif shadow_depth is not None:
            line = re.sub(r"\bb\.(?=[xyz]\b)", "bary_.", line)
        depth += line.count("{") - line.count("}")
        if shadow_depth is not None and depth < shadow_depth:
            shadow_depth = None
        out.append(line)
    body = "\n".join(out)
    text = "#undef FLT_MAX\nnamespace sh_%s {\nusing namespace glsl;\n%s\n}  // namespace sh_%s\n" % (name, body, name)
    for d in defines:
        text += "#undef %s\n" % d
    text += "#define FLT_MAX __FLT_MAX__\n"
    return text


def run(cmd, stdin_text=None):
    p = subprocess.run(cmd, input=stdin_text, text=True, capture_output=True)
    if p.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + p.stdout + p.stderr)
        raise SystemExit(1)


def main():
    if not os.path.isdir(os.path.join(REF, "Src")):
        print("reference tree not found at %s; oracle/_ref not built" % REF)
        return 1
    os.makedirs(OBJ, exist_ok=True)
    src = os.path.join(REF, "Src")
    inc = ["-I" + src, "-I" + os.path.join(REF, "3rdParty", "glad", "include"), "-I" + HERE]
    shim = ["-include", os.path.join(HERE, "ref_shim.h")]
    objs = []

    # Src/bvh.cpp:113 reads aabbRightSide[15] of a 15-element array on the
    # sweep's last step (all triangles left, right side empty).  g++ -O2 turns
    # that undefined read into a crash, so the array is given its 16th element
    # (an empty box, default-constructed): the step's cost becomes
    # n * area + 0 * inf = NaN and it never wins, which is the behaviour the
    # oracle restatement defines.  Nothing else in the file changes.
    with open(os.path.join(src, "bvh.cpp")) as fh:
        bvh = fh.read()
    assert bvh.count("BucketAABB aabbRightSide[15];") == 1
    bvh = "#line 1 \"%s\"\n" % os.path.join(src, "bvh.cpp") + bvh.replace(
        "BucketAABB aabbRightSide[15];", "BucketAABB aabbRightSide[16];")
    o = os.path.join(OBJ, "bvh.o")
    run(CXX + shim + inc + ["-x", "c++", "-c", "-", "-o", o], bvh)
    objs.append(o)

    o = os.path.join(OBJ, "compute.o")
    run(CXX + shim + inc + ["-c", os.path.join(src, "compute.cpp"), "-o", o])
    objs.append(o)

    with open(os.path.join(src, "mesh.cpp")) as fh:
        lines = fh.read().split("\n")
    part = "#include \"mesh.h\"\n#include <map>\n#include <tuple>\n#include <cassert>\n"
    part += "\n".join(lines[37:41]) + "\n" + "\n".join(lines[618:768]) + "\n"
    o = os.path.join(OBJ, "mesh_part.o")
    run(CXX + shim + inc + ["-x", "c++", "-c", "-", "-o", o], part)
    objs.append(o)

    # the loaders: includes, then everything between the Vector3 ordering and
    # the generators; the two rewrites only make MSVC-accepted code compile
    mesh_cpp = os.path.join(src, "mesh.cpp")
    loader = "#line 1 \"%s\"\n" % mesh_cpp + "\n".join(lines[0:37]) + "\n#line 42 \"%s\"\n" % mesh_cpp + \
        "\n".join(lines[41:617]) + "\n"
    for old, new in (("std::find_if(begin, end, std::isspace)", "std::find_if(begin, end, ::isspace)"),
                     ("auto &get_face_vertex_idx =", "auto get_face_vertex_idx =")):
        assert loader.count(old) == 1, old
        loader = loader.replace(old, new)
    tiny = os.path.join(REF, "3rdParty", "tinyply")
    o = os.path.join(OBJ, "mesh_loaders.o")
    run(CXX + shim + inc + ["-I" + tiny, "-x", "c++", "-c", "-", "-o", o], loader)
    objs.append(o)
    o = os.path.join(OBJ, "tinyply.o")
    run(CXX + ["-c", os.path.join(tiny, "tinyply.cpp"), "-o", o])
    objs.append(o)
    o = os.path.join(OBJ, "glad.o")
    run(["gcc", "-O2", "-fPIC", "-w", "-I" + os.path.join(REF, "3rdParty", "glad", "include"), "-c",
         os.path.join(REF, "3rdParty", "glad", "glad.c"), "-o", o])
    objs.append(o)

    o = os.path.join(OBJ, "image.o")
    run(CXX + shim + inc + ["-I" + os.path.join(REF, "3rdParty", "tinyexr"),
                            "-DexportNormalImage=ref_exportNormalImage", "-c", os.path.join(src, "image.cpp"), "-o", o])
    objs.append(o)

    o = os.path.join(OBJ, "tinyexr.o")
    run(CXX + ["-c", os.path.join(REF, "3rdParty", "tinyexr", "tinyexr.cc"), "-o", o])
    objs.append(o)

    o = os.path.join(OBJ, "host_driver.o")
    run(CXX + shim + inc + ["-I" + os.path.join(REF, "3rdParty", "tinyexr"),
                            "-c", os.path.join(HERE, "ref_host_driver.cpp"), "-o", o])
    objs.append(o)

    tu = "#include \"ref_glsl.h\"\n"
    for name in SHADERS:
        with open(os.path.join(REF, "Shaders", name + ".comp")) as fh:
            tu += glsl_to_cpp(fh.read(), name)
    tu += "#include \"ref_shader_driver.inc\"\n"
    o = os.path.join(OBJ, "shaders.o")
    run(CXX + ["-I" + HERE, "-x", "c++", "-c", "-", "-o", o], tu)
    objs.append(o)

    lib = os.path.join(OUT, "libfornos_ref.so")
    run(CXX + ["-shared", "-o", lib] + objs + ["-ldl"])
    print("built", lib)
    return 0


if __name__ == "__main__":
    sys.exit(main())
