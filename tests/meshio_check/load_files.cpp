// Loads every file named on the command line through fk_mesh_load (the
// library's OBJ / PLY readers, fornos_b200/csrc/fk_meshio.cpp, compiled here
// without the rest of the library) and prints how many loaded and how many
// were rejected.  The meshio tests build it under AddressSanitizer / UBSan
// and feed it mutated files.
#include <cstdio>

#include "../../fornos_b200/csrc/fk_internal.h"

int main(int argc, char** argv) {
  int loaded = 0, rejected = 0;
  for (int i = 1; i < argc; ++i) {
    fk_mesh* m = nullptr;
    if (fk_mesh_load(argv[i], &m) == FK_OK && m) {
      ++loaded;
      fk_mesh_free(m);
    } else {
      ++rejected;
    }
  }
  std::printf("loaded %d rejected %d\n", loaded, rejected);
  return 0;
}
