// kfun3d_meshgen: the seeded Kuhn-box mesh generator (kfun3d_mesh_generate in
// msh_io.cpp) as a stand-alone host program, so that a process which only
// needs an input mesh -- the timed CPU reference run of the benchmark -- does
// not load the CUDA library.
//
//   kfun3d_meshgen PATH N [BUMP_HEIGHT [SEED [JITTER [PERMUTE]]]]
//
// Defaults as kfun3d_mesh_spec's: bump 0.1, seed 0, jitter 0.2, permute 1,
// bump sigma 0.15.  Exit status 0 on success.
#include <cstdio>
#include <cstdlib>

#include "kfun3d_b200.h"
#include "internal.h"

// The generator reports failures through kf_set_error; the program prints them.
void kf_set_error(int code, const char *msg) { std::fprintf(stderr, "kfun3d_meshgen: error %d: %s\n", code, msg); }

// msh_io.cpp also holds the GEOMETRY loader, which this program never calls;
// its references to the matrix handle and the free stream resolve to these.
extern "C" void *CXX_Matrix_Init(const size_t, const size_t, const unsigned int, const unsigned int,
                                 const unsigned int *, const unsigned int *)
{
  return nullptr;
}
extern "C" void CXX_Matrix_Delete(void *) {}
extern "C" void kfun3d_get_freestream(double *u, double *v)
{
  *u = 1.0;
  *v = 0.0;
}

int main(int argc, char **argv)
{
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s PATH N [BUMP_HEIGHT [SEED [JITTER [PERMUTE]]]]\n", argv[0]);
    return 2;
  }
  kfun3d_mesh_spec s;
  s.n = std::atoi(argv[2]);
  s.bump_height = argc > 3 ? std::atof(argv[3]) : 0.1;
  s.bump_sigma = 0.15;
  s.jitter = argc > 5 ? std::atof(argv[5]) : 0.2;
  s.seed = argc > 4 ? std::strtoull(argv[4], nullptr, 10) : 0;
  s.permute = argc > 6 ? std::atoi(argv[6]) : 1;
  const int rc = kfun3d_mesh_generate(argv[1], &s);
  if (rc != 0) std::fprintf(stderr, "kfun3d_meshgen: kfun3d_mesh_generate returned %d\n", rc);
  return rc == 0 ? 0 : 1;
}
