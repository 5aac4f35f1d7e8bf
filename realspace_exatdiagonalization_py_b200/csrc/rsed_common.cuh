// Shared device helpers for the symmetry-resolved exact-diagonalization kernels.
//
// Bitmask convention (reference: utils/bitwise_operations.py:1-34): bit i-1 of a
// uint64 mask is site i (1-based sites); all masks of one catalog hold exactly
// n_filled set bits and n_site <= 63.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/rsed.h"

#define RSED_MAX_SITES 63
#define RSED_MAX_GROUP 64

// One entry of the representative table, indexed by the combinadic rank of a
// fixed-filling mask.  Same 16 bytes per state as the reference's three
// parallel tables (symmetry_resolved_ed.py:1359-1361): int32 representative
// index, int32 group element g with g(rep) = mask, complex64 amplitude alpha.
struct __align__(16) RsedEntry {
  int32_t rep;
  int32_t g;
  float re;
  float im;
};

// ---------------------------------------------------------------------------
// Combinadic (colexicographic) rank and unrank.
// rank(m) = sum_j C(b_j, j+1) over the set-bit positions b_0 < b_1 < ...
// (reference: symmetry_resolved_ed.py:122-140, 377-394).  `binom` is the
// (n_site+1) x (n_filled+1) row-major table C(b, j).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int64_t rsed_rank(uint64_t m, const int64_t* __restrict__ binom,
                                             int kp1) {
  int64_t r = 0;
  int j = 1;
  while (m) {
    int b = __ffsll((long long)m) - 1;
    r += binom[b * kp1 + j];
    ++j;
    m &= m - 1;
  }
  return r;
}

__device__ __forceinline__ uint64_t rsed_unrank(int64_t r, int n, int k,
                                                const int64_t* __restrict__ binom, int kp1) {
  uint64_t mask = 0;
  int b = n - 1;
  for (int j = k; j >= 1; --j) {
    while (binom[b * kp1 + j] > r) --b;
    mask |= 1ull << b;
    r -= binom[b * kp1 + j];
    --b;
  }
  return mask;
}

// ---------------------------------------------------------------------------
// Two-species bases: the sites in species_b hold exactly n_filled_b of the
// particles, the other sites the rest (e.g. spin up / spin down at fixed
// N_up, N_down).  Each species is ranked in colex order over its own sites in
// ascending order, and rank = rank_A * C(|B|, n_filled_b) + rank_B; the
// representative of an orbit is still its smallest mask.
// ---------------------------------------------------------------------------
struct RsedSpecies {
  uint64_t sb, sa;  // site masks of species B and A
  int kb, ka, nb, na;
  int64_t cb;       // C(nb, kb)
};

__device__ __forceinline__ RsedSpecies rsed_species(uint64_t sb, int n_site, int n_filled, int kb,
                                                    const int64_t* __restrict__ binom, int kp1) {
  RsedSpecies s;
  const uint64_t all = (n_site >= 64) ? ~0ull : ((1ull << n_site) - 1ull);
  s.sb = sb;
  s.sa = all & ~sb;
  s.kb = kb;
  s.ka = n_filled - kb;
  s.nb = __popcll(sb);
  s.na = n_site - s.nb;
  s.cb = binom[s.nb * kp1 + kb];
  return s;
}

__device__ __forceinline__ int64_t rsed_rank2(uint64_t m, const int64_t* __restrict__ binom, int kp1,
                                              uint64_t sb, int64_t cb) {
  int64_t ra = 0, rb = 0;
  int ja = 1, jb = 1;
  while (m) {
    const int b = __ffsll((long long)m) - 1;
    const int below_b = __popcll(sb & ((1ull << b) - 1ull));
    if ((sb >> b) & 1ull) {
      rb += binom[below_b * kp1 + jb];
      ++jb;
    } else {
      ra += binom[(b - below_b) * kp1 + ja];
      ++ja;
    }
    m &= m - 1;
  }
  return ra * cb + rb;
}

// rank for either basis kind (sb == 0: one species)
__device__ __forceinline__ int64_t rsed_rank_any(uint64_t m, const int64_t* __restrict__ binom, int kp1,
                                                 uint64_t sb, int64_t cb) {
  return sb ? rsed_rank2(m, binom, kp1, sb, cb) : rsed_rank(m, binom, kp1);
}

// Place bit p of `compact` at the p-th set bit of `sel` (ascending).
__device__ __forceinline__ uint64_t rsed_deposit(uint64_t compact, uint64_t sel) {
  uint64_t out = 0;
  for (uint64_t s = sel; s && compact; s &= s - 1, compact >>= 1)
    if (compact & 1ull) out |= s & (~s + 1ull);
  return out;
}

// Next mask with the same popcount (Gosper's hack; reference: :240-245).
__device__ __forceinline__ uint64_t rsed_gosper_next(uint64_t x) {
  uint64_t c = x & (~x + 1);
  uint64_t r = x + c;
  return (((r ^ x) >> 2) >> (__ffsll((long long)c) - 1)) | r;
}

// Image of mask m under the site permutation perm (0-based targets).
__device__ __forceinline__ uint64_t rsed_permute(uint64_t m, const uint8_t* __restrict__ perm) {
  uint64_t img = 0;
  while (m) {
    int b = __ffsll((long long)m) - 1;
    img |= 1ull << perm[b];
    m &= m - 1;
  }
  return img;
}

// Fermionic permutation parity of the occupied set: the number of occupied
// pairs whose order the permutation inverts, tracked as in the reference
// (symmetry_resolved_ed.py:303-309): for occupied sites in ascending order,
// count already-placed images above the current image.
__device__ __forceinline__ int rsed_perm_parity(uint64_t m, const uint8_t* __restrict__ perm) {
  uint64_t placed = 0;
  int par = 0;
  while (m) {
    int b = __ffsll((long long)m) - 1;
    int p = perm[b];
    par ^= __popcll(placed & ~((2ull << p) - 1ull)) & 1;
    placed |= 1ull << p;
    m &= m - 1;
  }
  return par;
}

// Total phase angle of U_g on mask m, summed exactly as the reference's byte
// tables do (symmetry_resolved_ed.py:346-374 then :538-542): per input byte a
// partial sum over its set bits in ascending order, then the byte partials
// added in ascending byte order.
__device__ __forceinline__ double rsed_angle_sum(uint64_t m, const double* __restrict__ ang,
                                                 int n_site) {
  double total = 0.0;
  for (int base = 0; base < n_site; base += 8) {
    unsigned v = (unsigned)((m >> base) & 0xFFu);
    if (v == 0u) {
      total = __dadd_rn(total, 0.0);
      continue;
    }
    double part = 0.0;
    while (v) {
      int i = __ffs(v) - 1;
      part = __dadd_rn(part, ang[base + i]);
      v &= v - 1u;
    }
    total = __dadd_rn(total, part);
  }
  return total;
}

// Complex product without FMA contraction, matching CPython/numpy's
// (ar*br - ai*bi, ar*bi + ai*br).
__device__ __forceinline__ double2 rsed_cmul_exact(double2 a, double2 b) {
  double2 r;
  r.x = __dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y));
  r.y = __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x));
  return r;
}

// Product-form phase of U_g on m (reference apply_operation_to_mask,
// symmetry_resolved_ed.py:977-1008): prod of eta_g(i) over occupied i in
// ascending order starting from 1+0j, times the fermionic parity.
__device__ __forceinline__ double2 rsed_phase_product(uint64_t m, const uint8_t* __restrict__ perm,
                                                      const double2* __restrict__ eta,
                                                      bool fermion, uint64_t* img_out) {
  double2 ph = make_double2(1.0, 0.0);
  uint64_t placed = 0;
  int par = 0;
  uint64_t t = m;
  while (t) {
    int b = __ffsll((long long)t) - 1;
    int p = perm[b];
    if (fermion) par ^= __popcll(placed & ~((2ull << p) - 1ull)) & 1;
    placed |= 1ull << p;
    ph = rsed_cmul_exact(ph, eta[b]);
    t &= t - 1;
  }
  if (fermion) {
    double s = par ? -1.0 : 1.0;
    ph = rsed_cmul_exact(ph, make_double2(s, 0.0));
  }
  *img_out = placed;
  return ph;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Per-thread error reporting: the first failing check stores its code.
__device__ __forceinline__ void rsed_flag_error(int* err, int code) {
  if (err) atomicCAS(err, 0, code);
}
