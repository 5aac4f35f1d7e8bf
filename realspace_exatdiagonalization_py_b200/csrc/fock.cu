// K9: sector state -> Fock amplitudes.
//
// A sector vector c (one coefficient per representative of the sector) is
// the state sum_col c_col / sqrt(|G| |Stab(s_col)|) sum_g conj(chi(g)) U_g |s_col>.
// One thread per basis state m (table rank r): the table gives m's
// representative s and one g with g(s) = m; the thread sums, in ascending g
// like the reference's dictionary accumulation, every group element that maps
// s to m, with the product-form phase U_g|s> = phase * |g s>.  Amplitudes at or
// below atol are dropped, the norm of the rest is summed per block, and a
// last pass rescales to unit norm.
#include "rsed_internal.cuh"

namespace {

constexpr int kFT = 256;

__global__ void __launch_bounds__(kFT) k_fock_amps(rsed_group_t grp, const int4* __restrict__ table,
                                                   const uint64_t* __restrict__ repr_masks,
                                                   const uint64_t* __restrict__ stab_mask,
                                                   const double2* __restrict__ xo, const double2* __restrict__ chi,
                                                   double atol, double2* __restrict__ amp,
                                                   uint64_t* __restrict__ masks, double* __restrict__ block_norm2) {
  __shared__ double red[kFT / 32];
  const int64_t r = (int64_t)blockIdx.x * kFT + threadIdx.x;
  double n2 = 0.0;
  if (r < grp.n_states) {
    const int4 e = __ldg(table + r);
    double2 sum = make_double2(0.0, 0.0);
    uint64_t m = 0;
    if (e.x >= 0) {
      const uint64_t s = repr_masks[e.x];
      const double2 co = xo[e.x];
      const int N = grp.n_site;
      const double2* eta = reinterpret_cast<const double2*>(grp.eta);
      uint64_t img;
      rsed_phase_product(s, grp.perm + (int64_t)e.y * N, eta + (int64_t)e.y * N, grp.fermionic, &m);
      if (sqrt(co.x * co.x + co.y * co.y) > atol) {
        const double inv = 1.0 / sqrt((double)grp.n_group * (double)__popcll(stab_mask[e.x]));
        const double2 pref = make_double2(co.x * inv, co.y * inv);
        for (int g = 0; g < grp.n_group; ++g) {
          const double2 ph = rsed_phase_product(s, grp.perm + (int64_t)g * N, eta + (int64_t)g * N, grp.fermionic,
                                                &img);
          if (img != m) continue;
          const double2 ch = chi[g];
          const double2 t = rsed_cmul_exact(rsed_cmul_exact(pref, make_double2(ch.x, -ch.y)), ph);
          sum = make_double2(sum.x + t.x, sum.y + t.y);
        }
        if (sqrt(sum.x * sum.x + sum.y * sum.y) <= atol) sum = make_double2(0.0, 0.0);
      }
    }
    amp[r] = sum;
    if (masks) masks[r] = m;
    n2 = sum.x * sum.x + sum.y * sum.y;
  }
  for (int o = 16; o > 0; o >>= 1) n2 += __shfl_xor_sync(0xffffffffu, n2, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = n2;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kFT / 32; ++w) t += red[w];
    block_norm2[blockIdx.x] = t;
  }
}

// One block: the block norms in order, then 1/sqrt into slot 0 of `out`.
__global__ void __launch_bounds__(kFT) k_fock_norm(const double* __restrict__ block_norm2, int64_t n_blocks,
                                                   double* __restrict__ out) {
  __shared__ double red[kFT];
  double t = 0.0;
  for (int64_t i = threadIdx.x; i < n_blocks; i += kFT) t += block_norm2[i];
  red[threadIdx.x] = t;
  __syncthreads();
  for (int w = kFT / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = red[0];
}

__global__ void k_fock_scale(double2* __restrict__ amp, int64_t n, const double* __restrict__ norm2) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const double inv = 1.0 / sqrt(norm2[0]);
  const double2 a = amp[r];
  amp[r] = make_double2(a.x * inv, a.y * inv);
}

}  // namespace

extern "C" size_t rsed_fock_scratch_bytes(int64_t n_states) {
  const int64_t n_blocks = (n_states + kFT - 1) / kFT;
  return sizeof(double) * (size_t)(n_blocks + 2);
}

extern "C" int rsed_fock_expand(const rsed_group_t* grp, const rsed_entry_t* table, int64_t n_orbits,
                                const uint64_t* repr_masks, const uint64_t* stab_mask, const double* x_orbit,
                                const double* chi, double atol, double* amp, uint64_t* masks, double* norm2_out,
                                void* scratch, size_t scratch_bytes, void* stream_) {
  int rc = check_group(grp);
  if (rc) return rc;
  RSED_REQUIRE(table && repr_masks && stab_mask && x_orbit && chi && amp && norm2_out && scratch && n_orbits >= 1,
               RSED_EINVAL, "bad Fock expansion arguments");
  RSED_REQUIRE(grp->eta != nullptr, RSED_EINVAL, "Fock expansion needs the group's eta phases");
  RSED_REQUIRE(scratch_bytes >= rsed_fock_scratch_bytes(grp->n_states), RSED_ESCRATCH, "Fock scratch too small");
  cudaStream_t stream = as_stream(stream_);
  const int64_t n_blocks = (grp->n_states + kFT - 1) / kFT;
  double* bn = reinterpret_cast<double*>(scratch);
  double* nrm = bn + n_blocks;
  k_fock_amps<<<(unsigned)n_blocks, kFT, 0, stream>>>(
      *grp, reinterpret_cast<const int4*>(table), repr_masks, stab_mask, reinterpret_cast<const double2*>(x_orbit),
      reinterpret_cast<const double2*>(chi), atol, reinterpret_cast<double2*>(amp), masks, bn);
  RSED_CHECK_LAUNCH();
  k_fock_norm<<<1, kFT, 0, stream>>>(bn, n_blocks, nrm);
  RSED_CHECK_LAUNCH();
  RSED_TRY_CUDA(cudaMemcpyAsync(norm2_out, nrm, sizeof(double), cudaMemcpyDeviceToHost, stream));
  RSED_TRY_CUDA(cudaStreamSynchronize(stream));
  RSED_REQUIRE(*norm2_out > atol, RSED_EINVAL, "Expanded state has near-zero norm.");
  k_fock_scale<<<(unsigned)((grp->n_states + 255) / 256), 256, 0, stream>>>(reinterpret_cast<double2*>(amp),
                                                                           grp->n_states, nrm);
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}

// ---- overlaps of dense Fock-amplitude vectors ---------------------------------
//
// states: complex128 [slot][level][rank], n_m levels of n_states amplitudes per
// slot.  For every pair p = (a, b) of slots, out[p][i][j] = sum_r
// conj(states[a][i][r]) * states[b][j][r].
//
// Work unit = (chunk of kOvChunk ranks, pair, T x T tile of (i, j)), T =
// min(n_m, 4), so a one- or two-state manifold keeps few registers and many
// warps in flight.  Units are numbered chunk-major, and one wave of blocks
// (occupancy x SMs) walks them with a grid stride, so the blocks in flight
// work on the same few chunks for every pair: a slot that several pairs share
// (each state of a Chern row enters up to four links) is read from DRAM once
// and from L2 after that.  Per unit a block streams the chunk with coalesced
// 16-byte loads (two ranks per thread and step for T <= 2), reduces, and
// writes the unit's T*T partial sums.  A second pass (one warp per output)
// adds the chunk partials in a fixed order.  The chunking does not depend on
// the device or the grid, so the result is the same on every run.
namespace {

constexpr int kOvT = 256;
constexpr int kOvMaxTile = 4;
constexpr int64_t kOvChunk = 4096;

struct OvShape {
  int64_t n_chunks;
  int n_tiles, tile;
  int64_t n_units;
};

OvShape ov_shape(int64_t n_states, int n_m, int n_pairs) {
  OvShape s;
  s.tile = n_m < kOvMaxTile ? n_m : kOvMaxTile;
  s.n_tiles = (n_m + s.tile - 1) / s.tile;
  s.n_chunks = (n_states + kOvChunk - 1) / kOvChunk;
  s.n_units = s.n_chunks * n_pairs * s.n_tiles * s.n_tiles;
  return s;
}

size_t ov_pairs_bytes(int n_pairs) { return ((size_t)n_pairs * 2 * sizeof(int32_t) + 255) / 256 * 256; }

template <int T>
__device__ __forceinline__ void ov_accumulate(const double2* __restrict__ A, const double2* __restrict__ B,
                                              int64_t n_states, int64_t r, int ni, int nj, double (&re)[T][T],
                                              double (&im)[T][T]) {
  double2 a[T], b[T];
#pragma unroll
  for (int i = 0; i < T; ++i) a[i] = i < ni ? __ldg(A + (int64_t)i * n_states + r) : make_double2(0.0, 0.0);
#pragma unroll
  for (int j = 0; j < T; ++j) b[j] = j < nj ? __ldg(B + (int64_t)j * n_states + r) : make_double2(0.0, 0.0);
#pragma unroll
  for (int i = 0; i < T; ++i)
#pragma unroll
    for (int j = 0; j < T; ++j) {
      re[i][j] = fma(a[i].x, b[j].x, fma(a[i].y, b[j].y, re[i][j]));
      im[i][j] = fma(a[i].x, b[j].y, fma(-a[i].y, b[j].x, im[i][j]));
    }
}

template <int T>
__global__ void __launch_bounds__(kOvT, T <= 2 ? 4 : 2) k_fock_overlap_part(const double2* __restrict__ states, int64_t n_states,
                                                            int n_m, const int32_t* __restrict__ pairs,
                                                            int n_tiles, int64_t n_chunks, int64_t n_units,
                                                            double2* __restrict__ part) {
  __shared__ double2 red[kOvT / 32][T * T];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t slot = (int64_t)n_m * n_states;
  const int tt2 = n_tiles * n_tiles;
  const int64_t per_chunk = n_units / n_chunks;  // pairs x tiles
  for (int64_t u = blockIdx.x; u < n_units; u += gridDim.x) {
    // unit u = chunk * (n_pairs * n_tiles^2) + p * n_tiles^2 + t
    const int64_t chunk = u / per_chunk;
    const int64_t p = (u % per_chunk) / tt2;
    const int t = (int)(u % tt2);
    const int ti0 = (t / n_tiles) * T, tj0 = (t % n_tiles) * T;
    const int ni = min(T, n_m - ti0), nj = min(T, n_m - tj0);
    const double2* A = states + (int64_t)pairs[2 * p] * slot + (int64_t)ti0 * n_states;
    const double2* B = states + (int64_t)pairs[2 * p + 1] * slot + (int64_t)tj0 * n_states;
    double re[T][T], im[T][T];
#pragma unroll
    for (int i = 0; i < T; ++i)
#pragma unroll
      for (int j = 0; j < T; ++j) re[i][j] = im[i][j] = 0.0;
    const int64_t r0 = chunk * kOvChunk;
    const int64_t r1 = min(n_states, r0 + kOvChunk);
    int64_t r = r0 + threadIdx.x;
    if (T <= 2) {
      for (; r + kOvT < r1; r += 2 * kOvT) {
        ov_accumulate<T>(A, B, n_states, r, ni, nj, re, im);
        ov_accumulate<T>(A, B, n_states, r + kOvT, ni, nj, re, im);
      }
    }
    for (; r < r1; r += kOvT) ov_accumulate<T>(A, B, n_states, r, ni, nj, re, im);
#pragma unroll
    for (int i = 0; i < T; ++i)
#pragma unroll
      for (int j = 0; j < T; ++j) {
        double x = re[i][j], y = im[i][j];
        for (int o = 16; o > 0; o >>= 1) {
          x += __shfl_xor_sync(0xffffffffu, x, o);
          y += __shfl_xor_sync(0xffffffffu, y, o);
        }
        if (lane == 0) red[warp][i * T + j] = make_double2(x, y);
      }
    __syncthreads();
    if (threadIdx.x < T * T) {
      double2 s = make_double2(0.0, 0.0);
      for (int w = 0; w < kOvT / 32; ++w) s = make_double2(s.x + red[w][threadIdx.x].x, s.y + red[w][threadIdx.x].y);
      part[u * (T * T) + threadIdx.x] = s;
    }
    __syncthreads();  // red is rewritten by the next unit
  }
}

// One warp per output: lane l adds the partials of chunks l, l + 32, ... in
// order, then a fixed butterfly combines the lanes.
__global__ void k_fock_overlap_final(const double2* __restrict__ part, int n_m, int tile, int n_tiles,
                                     int64_t n_chunks, int64_t per_chunk, int64_t n_out, double2* __restrict__ out) {
  const int64_t idx = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (idx >= n_out) return;  // whole warps leave together
  const int64_t mm = (int64_t)n_m * n_m;
  const int64_t p = idx / mm;
  const int i = (int)((idx % mm) / n_m), j = (int)(idx % n_m);
  const int t = (i / tile) * n_tiles + j / tile;
  const int tt = tile * tile;
  const int k = (i % tile) * tile + j % tile;
  const double2* src = part + (p * n_tiles * n_tiles + t) * tt + k;
  double x = 0.0, y = 0.0;
  for (int64_t c = lane; c < n_chunks; c += 32) {
    const double2 v = src[c * per_chunk * tt];
    x += v.x;
    y += v.y;
  }
  for (int o = 16; o > 0; o >>= 1) {
    x += __shfl_xor_sync(0xffffffffu, x, o);
    y += __shfl_xor_sync(0xffffffffu, y, o);
  }
  if (lane == 0) out[idx] = make_double2(x, y);
}

template <int T>
int ov_launch(const double2* st, int64_t n_states, int n_m, const int32_t* dpairs, const OvShape& s, double2* part,
              cudaStream_t stream) {
  int dev = 0, n_sm = 0, per_sm = 0;
  RSED_TRY_CUDA(cudaGetDevice(&dev));
  RSED_TRY_CUDA(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
  RSED_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fock_overlap_part<T>, kOvT, 0));
  int64_t grid = (int64_t)n_sm * (per_sm > 0 ? per_sm : 1);
  if (grid > s.n_units) grid = s.n_units;
  k_fock_overlap_part<T><<<(unsigned)grid, kOvT, 0, stream>>>(st, n_states, n_m, dpairs, s.n_tiles, s.n_chunks,
                                                              s.n_units, part);
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}

}  // namespace

extern "C" size_t rsed_fock_overlap_scratch_bytes(int64_t n_states, int32_t n_m, int32_t n_pairs) {
  if (n_states < 1 || n_m < 1 || n_pairs < 1) return 0;
  const OvShape s = ov_shape(n_states, n_m, n_pairs);
  return ov_pairs_bytes(n_pairs) + sizeof(double2) * (size_t)s.tile * s.tile * (size_t)s.n_units;
}

extern "C" int rsed_fock_overlaps(const double* states, int64_t n_states, int32_t n_m, int32_t n_slots,
                                  const int32_t* pairs, int32_t n_pairs, double* out, void* scratch,
                                  size_t scratch_bytes, void* stream_) {
  RSED_REQUIRE(states && pairs && out && scratch, RSED_EINVAL, "null Fock overlap argument");
  RSED_REQUIRE(n_states >= 1 && n_m >= 1 && n_m <= 512 && n_slots >= 1 && n_pairs >= 1, RSED_EINVAL,
               "Fock overlap sizes out of range");
  for (int32_t p = 0; p < 2 * n_pairs; ++p)
    RSED_REQUIRE(pairs[p] >= 0 && pairs[p] < n_slots, RSED_EINVAL, "Fock overlap pair names a slot out of range");
  RSED_REQUIRE(scratch_bytes >= rsed_fock_overlap_scratch_bytes(n_states, n_m, n_pairs), RSED_ESCRATCH,
               "Fock overlap scratch too small");
  cudaStream_t stream = as_stream(stream_);
  const OvShape s = ov_shape(n_states, n_m, n_pairs);
  int32_t* dpairs = reinterpret_cast<int32_t*>(scratch);
  double2* part = reinterpret_cast<double2*>(reinterpret_cast<char*>(scratch) + ov_pairs_bytes(n_pairs));
  RSED_TRY_CUDA(cudaMemcpyAsync(dpairs, pairs, sizeof(int32_t) * 2 * (size_t)n_pairs, cudaMemcpyHostToDevice,
                                stream));
  const double2* st = reinterpret_cast<const double2*>(states);
  int rc;
  switch (s.tile) {
    case 1: rc = ov_launch<1>(st, n_states, n_m, dpairs, s, part, stream); break;
    case 2: rc = ov_launch<2>(st, n_states, n_m, dpairs, s, part, stream); break;
    case 3: rc = ov_launch<3>(st, n_states, n_m, dpairs, s, part, stream); break;
    default: rc = ov_launch<4>(st, n_states, n_m, dpairs, s, part, stream);
  }
  if (rc) return rc;
  const int64_t n_out = (int64_t)n_pairs * n_m * n_m;
  k_fock_overlap_final<<<(unsigned)((n_out + 3) / 4), 128, 0, stream>>>(
      part, n_m, s.tile, s.n_tiles, s.n_chunks, s.n_units / s.n_chunks, n_out, reinterpret_cast<double2*>(out));
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}

// ---- Resta position operator projected into a manifold (charge pump) -------------
//
// For orbit o with representative s the projected operator is diagonal:
// elem(o) = (1/|G|) sum_g chi_to(g) conj(chi_from(g)) z(g(s)), z(m) = the
// product over the occupied sites j of m (ascending) of site_phase[j]; an
// element with |elem| <= 1e-13 is dropped.  out[i][j] = sum_o
// conj(x_to[i][o]) elem(o) x_from[j][o] over the orbit-layout vectors.  Units
// = (chunk of kOvChunk orbits, T x T tile of (i, j)); elem is recomputed per
// tile (|G| permutations per orbit, cheap against the vector stream).
namespace {

__device__ __forceinline__ double2 pos_elem(uint64_t s, const rsed_group_t& grp, const double2* __restrict__ w,
                                            const double2* __restrict__ site_phase, double inv_ng) {
  double2 e = make_double2(0.0, 0.0);
  for (int g = 0; g < grp.n_group; ++g) {
    uint64_t m = rsed_permute(s, grp.perm + (int64_t)g * grp.n_site);
    double2 z = make_double2(1.0, 0.0);
    while (m) {
      const int j = __ffsll((long long)m) - 1;
      z = rsed_cmul_exact(z, site_phase[j]);
      m &= m - 1;
    }
    const double2 t = rsed_cmul_exact(w[g], z);
    e = make_double2(e.x + t.x, e.y + t.y);
  }
  e = make_double2(e.x * inv_ng, e.y * inv_ng);
  if (sqrt(e.x * e.x + e.y * e.y) <= 1e-13) e = make_double2(0.0, 0.0);
  return e;
}

template <int T>
__global__ void __launch_bounds__(kOvT, 2) k_position_part(rsed_group_t grp, int64_t n_orbits,
                                                           const uint64_t* __restrict__ repr_masks,
                                                           const double2* __restrict__ chi_to,
                                                           const double2* __restrict__ chi_from,
                                                           const double2* __restrict__ site_phase, double inv_ng,
                                                           const double2* __restrict__ x_to, int k_to,
                                                           const double2* __restrict__ x_from, int k_from,
                                                           int n_tiles, int64_t n_chunks, int64_t n_units,
                                                           double2* __restrict__ part) {
  __shared__ double2 red[kOvT / 32][T * T];
  __shared__ double2 sw[64];
  __shared__ double2 sph[64];
  // chi_to(g) * conj(chi_from(g)), the reference's product order
  for (int g = threadIdx.x; g < grp.n_group; g += kOvT)
    sw[g] = rsed_cmul_exact(chi_to[g], make_double2(chi_from[g].x, -chi_from[g].y));
  for (int j = threadIdx.x; j < grp.n_site; j += kOvT) sph[j] = site_phase[j];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int tt2 = n_tiles * n_tiles;
  for (int64_t u = blockIdx.x; u < n_units; u += gridDim.x) {
    const int64_t chunk = u / tt2;
    const int t = (int)(u % tt2);
    const int ti0 = (t / n_tiles) * T, tj0 = (t % n_tiles) * T;
    const int ni = min(T, k_to - ti0), nj = min(T, k_from - tj0);
    const double2* A = x_to + (int64_t)ti0 * n_orbits;
    const double2* B = x_from + (int64_t)tj0 * n_orbits;
    double re[T][T], im[T][T];
#pragma unroll
    for (int i = 0; i < T; ++i)
#pragma unroll
      for (int j = 0; j < T; ++j) re[i][j] = im[i][j] = 0.0;
    const int64_t r1 = min(n_orbits, (chunk + 1) * kOvChunk);
    for (int64_t o = chunk * kOvChunk + threadIdx.x; o < r1; o += kOvT) {
      double2 a[T], b[T];
      bool any = false;
#pragma unroll
      for (int i = 0; i < T; ++i) {
        a[i] = i < ni ? __ldg(A + (int64_t)i * n_orbits + o) : make_double2(0.0, 0.0);
        any |= (a[i].x != 0.0) | (a[i].y != 0.0);
      }
      if (!any) continue;  // orbit outside the target sector (or a zero row)
      bool anyb = false;
#pragma unroll
      for (int j = 0; j < T; ++j) {
        b[j] = j < nj ? __ldg(B + (int64_t)j * n_orbits + o) : make_double2(0.0, 0.0);
        anyb |= (b[j].x != 0.0) | (b[j].y != 0.0);
      }
      if (!anyb) continue;
      const double2 e = pos_elem(__ldg(repr_masks + o), grp, sw, sph, inv_ng);
#pragma unroll
      for (int j = 0; j < T; ++j) b[j] = rsed_cmul_exact(e, b[j]);
#pragma unroll
      for (int i = 0; i < T; ++i)
#pragma unroll
        for (int j = 0; j < T; ++j) {
          re[i][j] = fma(a[i].x, b[j].x, fma(a[i].y, b[j].y, re[i][j]));
          im[i][j] = fma(a[i].x, b[j].y, fma(-a[i].y, b[j].x, im[i][j]));
        }
    }
#pragma unroll
    for (int i = 0; i < T; ++i)
#pragma unroll
      for (int j = 0; j < T; ++j) {
        double x = re[i][j], y = im[i][j];
        for (int o = 16; o > 0; o >>= 1) {
          x += __shfl_xor_sync(0xffffffffu, x, o);
          y += __shfl_xor_sync(0xffffffffu, y, o);
        }
        if (lane == 0) red[warp][i * T + j] = make_double2(x, y);
      }
    __syncthreads();
    if (threadIdx.x < T * T) {
      double2 s = make_double2(0.0, 0.0);
      for (int wq = 0; wq < kOvT / 32; ++wq)
        s = make_double2(s.x + red[wq][threadIdx.x].x, s.y + red[wq][threadIdx.x].y);
      part[u * (T * T) + threadIdx.x] = s;
    }
    __syncthreads();
  }
}

// out[i][j] from the chunk partials, one warp per output (fixed order).
__global__ void k_position_final(const double2* __restrict__ part, int k_to, int k_from, int tile, int n_tiles,
                                 int64_t n_chunks, double2* __restrict__ out) {
  const int64_t idx = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (idx >= (int64_t)k_to * k_from) return;
  const int i = (int)(idx / k_from), j = (int)(idx % k_from);
  const int t = (i / tile) * n_tiles + j / tile;
  const int tt = tile * tile;
  const int64_t per_chunk = (int64_t)n_tiles * n_tiles;
  const double2* src = part + (int64_t)t * tt + (i % tile) * tile + j % tile;
  double x = 0.0, y = 0.0;
  for (int64_t c = lane; c < n_chunks; c += 32) {
    const double2 v = src[c * per_chunk * tt];
    x += v.x;
    y += v.y;
  }
  for (int o = 16; o > 0; o >>= 1) {
    x += __shfl_xor_sync(0xffffffffu, x, o);
    y += __shfl_xor_sync(0xffffffffu, y, o);
  }
  if (lane == 0) out[idx] = make_double2(x, y);
}

template <int T>
int pos_launch(const rsed_group_t& grp, int64_t n_orbits, const uint64_t* repr_masks, const double2* cto,
               const double2* cfrom, const double2* ph, double inv_ng, const double2* x_to, int k_to,
               const double2* x_from, int k_from, const OvShape& s, double2* part, cudaStream_t stream) {
  int dev = 0, n_sm = 0, per_sm = 0;
  RSED_TRY_CUDA(cudaGetDevice(&dev));
  RSED_TRY_CUDA(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
  RSED_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_position_part<T>, kOvT, 0));
  int64_t grid = (int64_t)n_sm * (per_sm > 0 ? per_sm : 1);
  if (grid > s.n_units) grid = s.n_units;
  k_position_part<T><<<(unsigned)grid, kOvT, 0, stream>>>(grp, n_orbits, repr_masks, cto, cfrom, ph, inv_ng, x_to,
                                                          k_to, x_from, k_from, s.n_tiles, s.n_chunks, s.n_units,
                                                          part);
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}

OvShape pos_shape(int64_t n_orbits, int k_to, int k_from) {
  const int k = k_to > k_from ? k_to : k_from;
  return ov_shape(n_orbits, k, 1);
}

}  // namespace

extern "C" size_t rsed_position_scratch_bytes(int64_t n_orbits, int32_t k_to, int32_t k_from) {
  if (n_orbits < 1 || k_to < 1 || k_from < 1) return 0;
  const OvShape s = pos_shape(n_orbits, k_to, k_from);
  return sizeof(double2) * (size_t)s.tile * s.tile * (size_t)s.n_units;
}

extern "C" int rsed_position_overlaps(const rsed_group_t* grp, int64_t n_orbits, const uint64_t* repr_masks,
                                      const double* chi_to, const double* chi_from, const double* site_phase,
                                      const double* x_to, int32_t k_to, const double* x_from, int32_t k_from,
                                      double* out, void* scratch, size_t scratch_bytes, void* stream_) {
  int rc = check_group(grp);
  if (rc) return rc;
  RSED_REQUIRE(repr_masks && chi_to && chi_from && site_phase && x_to && x_from && out && scratch, RSED_EINVAL,
               "null position-operator argument");
  RSED_REQUIRE(n_orbits >= 1 && k_to >= 1 && k_from >= 1 && k_to <= 512 && k_from <= 512, RSED_EINVAL,
               "position-operator sizes out of range");
  RSED_REQUIRE(scratch_bytes >= rsed_position_scratch_bytes(n_orbits, k_to, k_from), RSED_ESCRATCH,
               "position-operator scratch too small");
  cudaStream_t stream = as_stream(stream_);
  const OvShape s = pos_shape(n_orbits, k_to, k_from);
  double2* part = reinterpret_cast<double2*>(scratch);
  const double inv_ng = 1.0 / (double)grp->n_group;
  const double2* ct = reinterpret_cast<const double2*>(chi_to);
  const double2* cf = reinterpret_cast<const double2*>(chi_from);
  const double2* ph = reinterpret_cast<const double2*>(site_phase);
  const double2* xt = reinterpret_cast<const double2*>(x_to);
  const double2* xf = reinterpret_cast<const double2*>(x_from);
  switch (s.tile) {
    case 1: rc = pos_launch<1>(*grp, n_orbits, repr_masks, ct, cf, ph, inv_ng, xt, k_to, xf, k_from, s, part, stream); break;
    case 2: rc = pos_launch<2>(*grp, n_orbits, repr_masks, ct, cf, ph, inv_ng, xt, k_to, xf, k_from, s, part, stream); break;
    case 3: rc = pos_launch<3>(*grp, n_orbits, repr_masks, ct, cf, ph, inv_ng, xt, k_to, xf, k_from, s, part, stream); break;
    default: rc = pos_launch<4>(*grp, n_orbits, repr_masks, ct, cf, ph, inv_ng, xt, k_to, xf, k_from, s, part, stream);
  }
  if (rc) return rc;
  const int64_t n_out = (int64_t)k_to * k_from;
  k_position_final<<<(unsigned)((n_out + 3) / 4), 128, 0, stream>>>(part, k_to, k_from, s.tile, s.n_tiles,
                                                                   s.n_chunks, reinterpret_cast<double2*>(out));
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}
