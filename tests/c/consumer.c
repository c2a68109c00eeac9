/* A plain C consumer of include/rbmd_force.h, linked against librbmd_b200.so: the calls a
 * host-side MD driver makes in place of ExecutionNVT::ComputeAllForce
 * (rbmd/framework/run/ExecutionNVT.cpp:185-222) -- create from the reference's JSON keys, pair
 * coefficients, bind, then per step the host-buffer force call in the reference's Vec3f (float)
 * layout, status and energies, destroy.
 *
 *   consumer          error paths that need no GPU (create, malformed JSON, call order, destroy)
 *   consumer gpu N    additionally an LJ system of N atoms on a jittered simple-cubic lattice:
 *                     prints "force i fx fy fz" for every atom and "energy lj" on stdout
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime.h>

#include "rbmd_force.h"

static const char* kConfig =
    "{\"init_configuration\": {\"read_data\": {\"unit\": \"LJ\", \"atom_style\": \"atomic\"}},"
    " \"hyper_parameters\": {\"force_field\": {\"type\": \"LJ/CUT\"},"
    "                        \"neighbor\": {\"type\": \"VERLETLIST\", \"cut_off\": 2.5}},"
    " \"execution\": {\"ensemble\": \"NVE\", \"timestep\": 0.005, \"temperature\": [1.0, 1.0, 1.0]},"
    " \"precision\": \"fp32\"}";

#define EXPECT(cond, ...)                      \
  do {                                         \
    if (!(cond)) {                             \
      fprintf(stderr, "FAIL: " __VA_ARGS__);   \
      fprintf(stderr, "\n");                   \
      return 1;                                \
    }                                          \
  } while (0)

static int host_checks(void) {
  rbmd_box box = {{0, 0, 0}, {10, 10, 10}};
  rbmd_force* f = NULL;
  EXPECT(rbmd_force_create("{ not json", 1, &box, &f) == RBMD_ERR_CONFIG, "malformed JSON accepted");
  EXPECT(strlen(rbmd_last_error()) > 0, "no error message for malformed JSON");
  EXPECT(rbmd_force_create(kConfig, 1, &box, &f) == RBMD_OK && f, "create: %s", rbmd_last_error());
  const double eps = 1.0, sig = 1.0;
  EXPECT(rbmd_force_set_pair_coeffs(f, 1, &eps, &sig) == RBMD_OK, "pair coeffs");
  EXPECT(rbmd_force_compute(f, NULL) == RBMD_ERR_STATE, "compute before bind accepted");
  EXPECT(rbmd_force_bind(f, NULL) == RBMD_ERR_ARG, "bind(NULL) accepted");
  rbmd_force_destroy(f);
  printf("host ok\n");
  return 0;
}

static int gpu_run(int n_side) {
  const int64_t n = (int64_t)n_side * n_side * n_side;
  const double a = pow(1.0 / 0.8, 1.0 / 3.0), L = a * n_side;
  float* pos = (float*)malloc(sizeof(float) * 3 * n);
  float* frc = (float*)malloc(sizeof(float) * 3 * n);
  srand(7);
  for (int64_t i = 0; i < n; ++i) {
    const int64_t ix = i % n_side, iy = (i / n_side) % n_side, iz = i / ((int64_t)n_side * n_side);
    const int64_t c[3] = {ix, iy, iz};
    for (int d = 0; d < 3; ++d) {
      const double jit = 0.08 * ((double)rand() / RAND_MAX - 0.5);
      pos[3 * i + d] = (float)(a * (c[d] + 0.5) + jit);
    }
  }
  rbmd_box box = {{0, 0, 0}, {L, L, L}};
  rbmd_force* f = NULL;
  EXPECT(rbmd_force_create(kConfig, 1, &box, &f) == RBMD_OK, "create: %s", rbmd_last_error());
  const double eps = 1.0, sig = 1.0;
  EXPECT(rbmd_force_set_pair_coeffs(f, 1, &eps, &sig) == RBMD_OK, "pair coeffs");
  double *d_pos = NULL, *d_force = NULL;
  EXPECT(cudaMalloc((void**)&d_pos, sizeof(double) * 3 * n) == cudaSuccess, "cudaMalloc");
  EXPECT(cudaMalloc((void**)&d_force, sizeof(double) * 3 * n) == cudaSuccess, "cudaMalloc");
  rbmd_atoms_dev atoms;
  memset(&atoms, 0, sizeof atoms);
  atoms.n_atoms = n;
  atoms.n_replicas = 1;
  atoms.pos = d_pos;
  atoms.force = d_force;
  EXPECT(rbmd_force_bind(f, &atoms) == RBMD_OK, "bind: %s", rbmd_last_error());
  /* per MD step: host positions in, host forces out (Vec3f layout) */
  for (int step = 0; step < 2; ++step)
    EXPECT(rbmd_force_compute_host_f32(f, pos, frc, NULL) == RBMD_OK, "compute_host_f32: %s", rbmd_last_error());
  uint32_t flags = 0;
  EXPECT(rbmd_force_status(f, &flags, 0, NULL) == RBMD_OK && flags == 0, "status flags 0x%x", flags);
  rbmd_energy e;
  EXPECT(rbmd_force_energy(f, &e, NULL) == RBMD_OK, "energy");
  for (int64_t i = 0; i < n; ++i) printf("force %lld %.9g %.9g %.9g\n", (long long)i, frc[3 * i], frc[3 * i + 1], frc[3 * i + 2]);
  printf("energy %.12g\n", e.lj);
  rbmd_force_destroy(f);
  cudaFree(d_pos);
  cudaFree(d_force);
  free(pos);
  free(frc);
  return 0;
}

int main(int argc, char** argv) {
  if (host_checks()) return 1;
  if (argc > 1 && strcmp(argv[1], "gpu") == 0) return gpu_run(argc > 2 ? atoi(argv[2]) : 10);
  return 0;
}
