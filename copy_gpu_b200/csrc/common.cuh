// common.cuh -- device data layout and helpers shared by the sm_100a kernels.
//
// Layout in HBM (library-owned):
//   * atoms are binned into per-replica cell grids; the cell-sorted order ("slots") keeps
//     replicas contiguous because replica r's cells occupy [cell_base_r, cell_base_r + ncell_r);
//   * pos4[slot]  : Real4 (x, y, z, q)  -- position rounded to the compute precision + charge;
//   * frac[slot]  : fixed-point fractional coordinates (uint32 per axis for FP32, uint64 for
//                   FP64) + charge, the input of every k-space phase (exact integer phases);
//   * meta[slot]  : int2 (type, molecule);
//   * nbr[p * stride + slot] : neighbour entry (j_slot << 6 | shift code), transposed so that a
//                   warp of consecutive slots reads one 128-byte line per neighbour index.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace rbmd {

constexpr int kMaxReplicaTypes = 16;   // per-type LJ table lives in shared memory
constexpr int kMaxCellAtoms = 1024;    // cell rank-sort bound (RBMD_FLAG_CELL_OVERFLOW beyond)
constexpr int kShiftBits = 6;

// status bits (mirrors include/rbmd_force.h)
constexpr uint32_t kFlagListOverflow = 0x01u;
constexpr uint32_t kFlagCellOverflow = 0x02u;
constexpr uint32_t kFlagShakeNoConv = 0x04u;
constexpr uint32_t kFlagNonFinite = 0x08u;
constexpr uint32_t kFlagOutOfBox = 0x10u;
constexpr uint32_t kFlagSampler = 0x20u;
constexpr uint32_t kFlagShakeSingular = 0x40u;

struct RepDev {
  float lo_f[3], hi_f[3], box_f[3], dx_f[3], wrap_f[3];  // wrap_f = dx_f * dims (reference offset)
  double lo_d[3], hi_d[3], box_d[3], dx_d[3], wrap_d[3];
  int dims[3];
  int cell_base, ncell;
  int atom_begin, atom_end;
  int k_begin, P;
  double volume;
  double S;          // RBE normaliser prod_d H_d - 1
  double kT_target;  // thermostat target (kB * T0 units handled on host)
  int ndof_mode;     // unused on device
  int rbl_pice;      // RBL: every rbl_pice-th shell pair is kept and weighted by rbl_pice
};

template <class R> struct Traits;
template <> struct Traits<float> {
  using V4 = float4;
  static __device__ __forceinline__ float lo(const RepDev& r, int d) { return r.lo_f[d]; }
  static __device__ __forceinline__ float box(const RepDev& r, int d) { return r.box_f[d]; }
  static __device__ __forceinline__ float dx(const RepDev& r, int d) { return r.dx_f[d]; }
  static __device__ __forceinline__ float wrap(const RepDev& r, int d) { return r.wrap_f[d]; }
};
template <> struct Traits<double> {
  using V4 = double4;
  static __device__ __forceinline__ double lo(const RepDev& r, int d) { return r.lo_d[d]; }
  static __device__ __forceinline__ double box(const RepDev& r, int d) { return r.box_d[d]; }
  static __device__ __forceinline__ double dx(const RepDev& r, int d) { return r.dx_d[d]; }
  static __device__ __forceinline__ double wrap(const RepDev& r, int d) { return r.wrap_d[d]; }
};

struct Frac32 { uint32_t x, y, z; float q; };               // 16 B
struct Frac64 { unsigned long long x, y, z; double q; };     // 32 B

// Fixed-point turn of a fractional coordinate f in [0, 1]: floor(f * 2^32) (2^64).  f can round
// up to exactly 1.0 (f = u - floor(u) for u a hair below an integer); that is a whole turn and
// wraps to 0, as periodicity requires.  A NaN coordinate gives an unspecified turn (the status
// word's non-finite flag is raised by the force passes).
__host__ __device__ __forceinline__ uint32_t turn32(double f) {
  const double s = f * 4294967296.0;
  return s >= 4294967296.0 ? 0u : (uint32_t)s;
}
__host__ __device__ __forceinline__ unsigned long long turn64(double f) {
  const double s = f * 18446744073709551616.0;
  return s >= 18446744073709551616.0 ? 0ull : (unsigned long long)s;
}

// exact-rounding arithmetic (never contracted into FMA): used wherever the result must equal
// the oracle bit for bit (cell index, neighbour predicate)
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }

// Two-float compensated accumulator (Knuth's TwoSum: s + e == a + b exactly).  The per-atom
// force is kept as an unevaluated sum hi + lo; for Real=double it degrades to a plain sum.
template <class R> struct Acc {
  R hi = 0, lo = 0;
  __device__ __forceinline__ void add(R b) {
    R s = add_rn(hi, b);
    R bb = sub_rn(s, hi);
    R e = add_rn(sub_rn(hi, sub_rn(s, bb)), sub_rn(b, bb));
    hi = s;
    lo = add_rn(lo, e);
  }
  __device__ __forceinline__ double value() const { return (double)hi + (double)lo; }
};
template <> struct Acc<double> {
  double hi = 0;
  __device__ __forceinline__ void add(double b) { hi += b; }
  __device__ __forceinline__ double value() const { return hi; }
};

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), same stream as the oracle's.
__host__ __device__ __forceinline__ void philox4x32(uint32_t c[4], uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)M0 * c[0];
    uint64_t p1 = (uint64_t)M1 * c[2];
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
    k0 += W0;
    k1 += W1;
  }
}

__device__ __forceinline__ void set_flag(uint32_t* status, uint32_t f) { atomicOr(status, f); }

}  // namespace rbmd
