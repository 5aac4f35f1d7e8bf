// K6b: orbit-space projection table and its streaming SpMV.
//
// The on-the-fly apply (apply.cu) re-derives every hop on every call: gate
// test, combinadic rank, a random 16-B gather from the C(N,k)-sized table.
// Across the ~100 matvecs of one eigen-solve those hops never change, so this
// file builds them once per catalog state into a CSR over orbit rows whose
// entries carry only what does not depend on the sector:
//   cg = c | g << 26   (target orbit, group element)
//   w  = conj(t * s_JW * alpha) * sqrt(S_c) / sqrt(S_r)
// A matvec then streams the table from HBM once per column chunk and gathers
// x[c][chunk] rows; chunks are sized by the caller so that x[:, chunk] stays
// resident in L2 while the table streams past it.
#include <type_traits>
#include "rsed_internal.cuh"
#include "rsed_apply.cuh"

using namespace rsed_apply;

namespace {

constexpr int kOrbitBits = 26;
constexpr uint32_t kOrbitMask = (1u << kOrbitBits) - 1u;

// Hops of row r in the order of the on-the-fly apply: occupied source site
// ascending, then the terms of that site in order, skipping occupied targets.
__global__ void __launch_bounds__(256) k_proj_count(rsed_model_t md, int64_t* counts, ApplySmemLayout lay) {
  extern __shared__ __align__(16) unsigned char smem[];
  rsed_sectors_t none{};
  ApplyView v = stage_apply(md, none, lay, smem);
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= md.n_orbits) return;
  const uint64_t m = md.repr_masks[r];
  int64_t n = 0;
  uint64_t occ = m;
  while (occ) {
    const int i = __ffsll((long long)occ) - 1;
    occ &= occ - 1;
    for (int t = v.tbeg[i]; t < v.tbeg[i + 1]; ++t) n += ((m >> v.tto[t]) & 1ull) ? 0 : 1;
  }
  counts[r] = n;
}

// Table entries are gathered HB hops at a time so each thread keeps several
// random 16-B loads in flight.
template <int HB>
__global__ void __launch_bounds__(256) k_proj_fill(rsed_model_t md, const double* __restrict__ sqrt_stab,
                                                   const int64_t* __restrict__ rowptr, uint32_t* __restrict__ cg,
                                                   double2* __restrict__ w64, float2* __restrict__ w32,
                                                   ApplySmemLayout lay) {
  extern __shared__ __align__(16) unsigned char smem[];
  rsed_sectors_t none{};
  ApplyView v = stage_apply(md, none, lay, smem);
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= md.n_orbits) return;
  const int kp1 = md.n_filled + 1;
  const int64_t cbs = md.species_b ? v.binom[__popcll(md.species_b) * kp1 + md.n_filled_b] : 1;
  const uint64_t m = md.repr_masks[r];
  const double sr = sqrt_stab[r];
  int64_t pos = rowptr[r];
  int bt[HB];
  int64_t bidx[HB];
  int nh = 0;
  auto flush = [&](int cnt) {
    RsedEntry e[HB];
#pragma unroll
    for (int h = 0; h < HB; ++h)
      if (h < cnt) e[h] = load_entry(reinterpret_cast<const RsedEntry*>(md.table), bidx[h]);
    double sq[HB];
#pragma unroll
    for (int h = 0; h < HB; ++h)
      if (h < cnt) sq[h] = __ldg(sqrt_stab + e[h].rep);
#pragma unroll
    for (int h = 0; h < HB; ++h) {
      if (h >= cnt) continue;
      const int t = bt[h];
      double2 ta = cmul(v.tamp[t], make_double2(e[h].re, e[h].im));
      if (md.fermionic && (__popcll(m & v.tjw[t]) & 1)) {
        ta.x = -ta.x;
        ta.y = -ta.y;
      }
      const double ratio = sq[h] / sr;
      const double2 w = make_double2(ta.x * ratio, -ta.y * ratio);
      if (cg) cg[pos] = (uint32_t)e[h].rep | ((uint32_t)e[h].g << kOrbitBits);
      if (w64) w64[pos] = w;
      if (w32) w32[pos] = make_float2((float)w.x, (float)w.y);
      ++pos;
    }
  };
  uint64_t occ = m;
  while (occ) {
    const int i = __ffsll((long long)occ) - 1;
    occ &= occ - 1;
    for (int t = v.tbeg[i]; t < v.tbeg[i + 1]; ++t) {
      const int jj = v.tto[t];
      if ((m >> jj) & 1ull) continue;
      bt[nh] = t;
      bidx[nh] = rsed_rank_any(m ^ (1ull << i) ^ (1ull << jj), v.binom, kp1, md.species_b, cbs);
      if (++nh == HB) {
        flush(HB);
        nh = 0;
      }
    }
  }
  if (nh) flush(nh);
}

// ---- streaming SpMV --------------------------------------------------------
// One warp per orbit row (grid-stride).  The warp's lanes form EPW = 32/L
// entry slots of L lanes; the L lanes of a slot cover the NC = L*CPL columns
// of the chunk, CPL contiguous columns each (one 16-B gather per lane and
// hop).  Entry slots walk the row's hops EPW at a time, U hops per batch
// (all U table entries, then all U x rows, then the arithmetic), and are
// summed with xor-shuffles at the end of the row.
template <int PREC>
struct ProjTypes;
template <>
struct ProjTypes<64> {
  using W = double2;
  using Real = double;
};
template <>
struct ProjTypes<32> {
  using W = float2;
  using Real = float;
};

// CPL contiguous columns of one x row, loaded as 16-B vectors (two FP32 or one
// FP64 complex value each); vectors at or beyond the row's leading dimension
// read as zero, so a lane's segment never leaves its row.
template <int PREC, int CPL>
struct XVec {
  using W = typename ProjTypes<PREC>::W;
  static constexpr int kPer = (PREC == 64) ? 1 : 2;  // columns per 16-B vector
  static constexpr int kVec = CPL / kPer;
  W v[CPL];
  __device__ __forceinline__ void load(const char* base, int avail) {
#pragma unroll
    for (int k = 0; k < kVec; ++k) {
      if (k * kPer < avail) {
        if constexpr (PREC == 64) {
          v[k] = __ldg(reinterpret_cast<const double2*>(base) + k);
        } else {
          const float4 q = __ldg(reinterpret_cast<const float4*>(base) + k);
          v[2 * k] = make_float2(q.x, q.y);
          v[2 * k + 1] = make_float2(q.z, q.w);
        }
      } else {
#pragma unroll
        for (int j = 0; j < kPer; ++j) v[k * kPer + j].x = v[k * kPer + j].y = 0;
      }
    }
  }
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int j = 0; j < CPL; ++j) v[j].x = v[j].y = 0;
  }
};

template <typename T>
__device__ __forceinline__ T ld_stream(const T* p) {
  return __ldcs(p);
}

// The hops of one row for an FP32 lane of 4 columns that form two sector
// pairs (columns 0-1 in sector s0, 2-3 in s2) when the row belongs to every
// sector of the warp: no per-column tests, one weight-character product per
// pair, and the table entries of the next batch loaded while the current
// batch gathers.  Missing entries past the row's end become (orbit 0,
// weight 0), so the loop body has no branches (x is finite: the solver's
// own Lanczos blocks).
template <int L, int U>
__device__ __forceinline__ void spmv_row_pairs32(const uint32_t* __restrict__ cgt, const float2* __restrict__ wt,
                                                 int64_t e0, int64_t e1, int eslot, const char* __restrict__ xl,
                                                 uint32_t rowb, const float2* ch0, const float2* ch2, int nsec,
                                                 float2 acc[4]) {
  constexpr int EPW = 32 / L;
  constexpr int B = EPW * U;  // hops per batch and warp
  float2 a0 = make_float2(0.f, 0.f), a1 = a0, a2 = a0, a3 = a0;
  uint32_t cgn[U];
  float2 wn[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const int64_t idx = e0 + u * EPW + eslot;
    const bool ok = idx < e1;
    cgn[u] = ok ? ld_stream(cgt + idx) : 0u;
    wn[u] = ok ? ld_stream(wt + idx) : make_float2(0.f, 0.f);
  }
  for (int64_t base = e0; base < e1; base += B) {
    uint32_t cgc[U];
    float2 wc[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      cgc[u] = cgn[u];
      wc[u] = wn[u];
    }
    if (base + B < e1) {
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int64_t idx = base + B + u * EPW + eslot;
        const bool ok = idx < e1;
        cgn[u] = ok ? ld_stream(cgt + idx) : 0u;
        wn[u] = ok ? ld_stream(wt + idx) : make_float2(0.f, 0.f);
      }
    }
    float4 xa[U], xc[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      // the lane's 32-B segment in one 256-bit load (32-B aligned: see the caller)
      const char* px = xl + (size_t)(cgc[u] & kOrbitMask) * rowb;
      asm("{\n\t.reg .u64 ga;\n\tcvta.to.global.u64 ga, %8;\n\t"
          "ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [ga];\n\t}"
          : "=f"(xa[u].x), "=f"(xa[u].y), "=f"(xa[u].z), "=f"(xa[u].w), "=f"(xc[u].x), "=f"(xc[u].y),
            "=f"(xc[u].z), "=f"(xc[u].w)
          : "l"(px));
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int go = (int)(cgc[u] >> kOrbitBits) * nsec;
      const float2 c0 = ch0[go], c2 = ch2[go];
      const float2 w = wc[u];
      const float p0x = w.x * c0.x - w.y * c0.y, p0y = w.x * c0.y + w.y * c0.x;
      const float p2x = w.x * c2.x - w.y * c2.y, p2y = w.x * c2.y + w.y * c2.x;
      a0.x += p0x * xa[u].x - p0y * xa[u].y;
      a0.y += p0x * xa[u].y + p0y * xa[u].x;
      a1.x += p0x * xa[u].z - p0y * xa[u].w;
      a1.y += p0x * xa[u].w + p0y * xa[u].z;
      a2.x += p2x * xc[u].x - p2y * xc[u].y;
      a2.y += p2x * xc[u].y + p2y * xc[u].x;
      a3.x += p2x * xc[u].z - p2y * xc[u].w;
      a3.y += p2x * xc[u].w + p2y * xc[u].z;
    }
  }
  acc[0] = a0;
  acc[1] = a1;
  acc[2] = a2;
  acc[3] = a3;
}

template <int PREC, int L, int CPL, int U>
__global__ void __launch_bounds__(256, 3) k_proj_spmv(rsed_model_t md, rsed_sectors_t sc, const void* __restrict__ xin,
                                                   double2* __restrict__ y, int chunk0) {
  using W = typename ProjTypes<PREC>::W;
  using Real = typename ProjTypes<PREC>::Real;
  constexpr int EPW = 32 / L;
  constexpr int NC = L * CPL;
  extern __shared__ __align__(16) unsigned char smem[];
  // characters transposed to [g][sector]: the L lanes of an entry slot share
  // g and read consecutive words
  W* chi = reinterpret_cast<W*>(smem);
  const double2* gchi = reinterpret_cast<const double2*>(sc.chi);
  const int nsec = sc.n_sectors;
  const int nchi = nsec * md.n_group;
  for (int i = threadIdx.x; i < nchi; i += blockDim.x) {
    const int s = i / md.n_group, g = i % md.n_group;
    const double2 c = gchi[i];
    chi[g * nsec + s].x = (Real)c.x;
    chi[g * nsec + s].y = (Real)c.y;
  }
  __syncthreads();
  const W* __restrict__ wt = reinterpret_cast<const W*>(PREC == 64 ? (const void*)md.proj_w64
                                                                    : (const void*)md.proj_w32);
  const uint32_t* __restrict__ cgt = md.proj_cg;
  const int64_t* __restrict__ rp = md.proj_rowptr;
  const int lane = threadIdx.x & 31;
  const int eslot = lane / L;
  const int c0 = (chunk0 + (int)blockIdx.y) * NC + (lane % L) * CPL;
  const int64_t ld = sc.ld;
  const int avail = (int)ld - c0;
  int sec[CPL];
  bool colv[CPL], fresh[CPL];
#pragma unroll
  for (int j = 0; j < CPL; ++j) {
    colv[j] = c0 + j < sc.n_cols;
    sec[j] = colv[j] ? sc.col_sector[c0 + j] : -1;
    // the block vectors of one sector sit in adjacent columns, so a lane's
    // columns usually share the hop weight
    fresh[j] = (j == 0) || sec[j] != sec[j - 1];
  }
  const char* xb = reinterpret_cast<const char*>(xin) + (size_t)c0 * sizeof(W);
  // FP32 lanes of 4 columns in two sector pairs (blocks of 2 or 4 columns):
  // the branch-free row loop whenever the row is in all of the warp's sectors.
  // Lanes past the last column run it too, on column 0 of x (in bounds), and
  // their sums are dropped.
  bool pairs = false;
  const char* xfast = xb;
  int s0 = 0, s2 = 0;
  if constexpr (PREC == 32 && CPL == 4) {
    // a lane's 4 columns start at a multiple of 4: with ld a multiple of 4 too
    // (and x 32-B aligned) each segment is 32-B aligned for one 256-bit load
    const bool lane_ok = colv[3] ? (sec[1] == sec[0] && sec[3] == sec[2]) : !colv[0];
    pairs = __all_sync(0xffffffffu, lane_ok) && (ld % 4) == 0 &&
            (reinterpret_cast<uintptr_t>(xin) & 31) == 0;
    if (!colv[0]) xfast = reinterpret_cast<const char*>(xin);
    s0 = colv[0] ? sec[0] : 0;
    s2 = colv[0] ? sec[2] : 0;
  }
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t r = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < md.n_orbits; r += warps) {
    const uint64_t memr = sc.member[r];
    bool on[CPL];
    bool any = false;
#pragma unroll
    for (int j = 0; j < CPL; ++j) {
      on[j] = colv[j] && ((memr >> sec[j]) & 1ull);
      any |= on[j];
    }
    W acc[CPL];
#pragma unroll
    for (int j = 0; j < CPL; ++j) acc[j].x = acc[j].y = (Real)0;
    bool done = false;
    if constexpr (PREC == 32 && CPL == 4) {
      if (pairs && __all_sync(0xffffffffu, !colv[0] || (on[0] && on[1] && on[2] && on[3]))) {
        const float2* chb = reinterpret_cast<const float2*>(chi);
        spmv_row_pairs32<L, U>(cgt, reinterpret_cast<const float2*>(wt), rp[r], rp[r + 1], eslot, xfast,
                               (uint32_t)(ld * sizeof(float2)), chb + s0, chb + s2, nsec,
                               reinterpret_cast<float2*>(acc));
        done = true;
      }
    }
    if (!done && __any_sync(0xffffffffu, any)) {
      const int64_t e0 = rp[r], e1 = rp[r + 1];
      for (int64_t base = e0; base < e1; base += EPW * U) {
        uint32_t cgv[U];
        W wv[U];
        XVec<PREC, CPL> xv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int64_t idx = base + u * EPW + eslot;
          if (idx < e1) {
            cgv[u] = ld_stream(cgt + idx);
            wv[u] = ld_stream(wt + idx);
          } else {
            cgv[u] = 0xffffffffu;
            wv[u].x = wv[u].y = (Real)0;
          }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          if (cgv[u] != 0xffffffffu && any)
            xv[u].load(xb + (size_t)(cgv[u] & kOrbitMask) * ld * sizeof(W), avail);
          else
            xv[u].zero();
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          if (cgv[u] == 0xffffffffu) continue;
          const W* chg = chi + (int)(cgv[u] >> kOrbitBits) * nsec;
          Real wcx = 0, wcy = 0;
#pragma unroll
          for (int j = 0; j < CPL; ++j) {
            if (!on[j]) continue;
            if (fresh[j] || !on[j - (j > 0)]) {
              const W ch = chg[sec[j]];
              wcx = wv[u].x * ch.x - wv[u].y * ch.y;
              wcy = wv[u].x * ch.y + wv[u].y * ch.x;
            }
            const W xx = xv[u].v[j];
            acc[j].x += wcx * xx.x - wcy * xx.y;
            acc[j].y += wcx * xx.y + wcy * xx.x;
          }
        }
      }
    }
#pragma unroll
    for (int off = L; off < 32; off <<= 1) {
#pragma unroll
      for (int j = 0; j < CPL; ++j) {
        acc[j].x += __shfl_xor_sync(0xffffffffu, acc[j].x, off);
        acc[j].y += __shfl_xor_sync(0xffffffffu, acc[j].y, off);
      }
    }
    if (eslot == 0) {
      const double2 hd = reinterpret_cast<const double2*>(md.hdiag)[r];
#pragma unroll
      for (int j = 0; j < CPL; ++j) {
        if (!colv[j]) continue;
        double2 o = make_double2(0.0, 0.0);
        if (on[j]) {
          const W xr = reinterpret_cast<const W*>(xin)[r * ld + c0 + j];
          const double xx = (double)xr.x, xy = (double)xr.y;
          o.x = (double)acc[j].x + (hd.x * xx + hd.y * xy);
          o.y = (double)acc[j].y + (hd.x * xy - hd.y * xx);
        }
        y[r * ld + c0 + j] = o;
      }
    }
  }
}

template <int PREC, int L, int CPL>
int launch_spmv(const rsed_model_t& md, const rsed_sectors_t& sc, const void* x, double2* y, bool sequential,
                cudaStream_t stream) {
  using W = typename ProjTypes<PREC>::W;
  constexpr int U = 4;
  constexpr int NC = L * CPL;
  auto kern = k_proj_spmv<PREC, L, CPL, U>;
  const size_t smem = sizeof(W) * (size_t)sc.n_sectors * md.n_group;
  static int blocks_per_sm[16] = {0};  // per device, computed once
  int dev = 0;
  RSED_TRY_CUDA(cudaGetDevice(&dev));
  int& bps = blocks_per_sm[dev & 15];
  if (smem > 48 * 1024)
    RSED_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  if (bps == 0) {
    RSED_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, 256, smem));
    if (bps < 1) bps = 1;
  }
  static int n_sm = 0;
  if (n_sm == 0) RSED_TRY_CUDA(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
  const int n_chunks = (sc.n_cols + NC - 1) / NC;
  const int64_t row_blocks = (md.n_orbits + 7) / 8;
  const int64_t gx = row_blocks < (int64_t)n_sm * bps ? row_blocks : (int64_t)n_sm * bps;
  if (sequential) {
    for (int c = 0; c < n_chunks; ++c) {
      kern<<<dim3((unsigned)gx, 1), 256, smem, stream>>>(md, sc, x, y, c);
      RSED_CHECK_LAUNCH();
    }
  } else {
    kern<<<dim3((unsigned)gx, (unsigned)n_chunks), 256, smem, stream>>>(md, sc, x, y, 0);
    RSED_CHECK_LAUNCH();
  }
  return RSED_OK;
}

int check_proj_model(const rsed_model_t* md) {
  RSED_REQUIRE(md != nullptr, RSED_EINVAL, "model descriptor is NULL");
  RSED_REQUIRE(md->n_site >= 1 && md->n_site <= RSED_MAX_SITES, RSED_ERANGE, "bad n_site");
  RSED_REQUIRE(md->n_group >= 1 && md->n_group <= RSED_MAX_GROUP, RSED_ERANGE, "bad |G|");
  RSED_REQUIRE(md->n_orbits >= 1 && md->table && md->repr_masks && md->binom && md->hdiag, RSED_EINVAL,
               "model tables missing");
  RSED_REQUIRE(md->n_terms >= 0 && md->term_begin, RSED_EINVAL, "terms missing");
  RSED_REQUIRE(md->n_orbits <= (int64_t)kOrbitMask, RSED_ERANGE,
               "projection table holds at most 2^26 - 1 orbits");
  return RSED_OK;
}

}  // namespace

// Called by rsed_apply_h for variants 0 (with a table present), 3NN-6NN.
int rsed_proj_apply(const rsed_model_t& md, const rsed_sectors_t& sc, const void* x, double2* y, int precision,
                    int variant, cudaStream_t stream) {
  RSED_REQUIRE(md.proj_rowptr && md.proj_cg, RSED_EINVAL, "no projection table in the model");
  RSED_REQUIRE(precision == 64 ? md.proj_w64 != nullptr : md.proj_w32 != nullptr, RSED_EINVAL,
               "projection table has no weights for precision %d", precision);
  RSED_REQUIRE((sc.ld & 1) == 0 && (reinterpret_cast<uintptr_t>(x) & 15) == 0, RSED_EINVAL,
               "projection apply needs an even leading dimension and a 16-byte aligned x");
  if (variant == 0) {
    // Measured on B200 (657,756 orbits, 64 columns): FP32 runs best with a
    // 32-B x segment per lane (4 columns) and one chunk covering up to 64
    // columns (3.7 ms vs 4.5 ms with 16-B segments; at 32 columns 1.48 ms in
    // one chunk vs 1.95 ms in chunks of 16 that keep x in L2); FP64 with
    // 16-B segments and 16-column chunks, one after another (7.5 ms; wider
    // segments spill into lower occupancy), except at 17-32 columns.  Small (latency-bound) bases prefer 16 columns
    // per chunk with all chunks in one launch, for more warps in flight.
    if (md.n_orbits < 65536) {
      variant = 416;
    } else if (precision == 32) {
      int nc = 8;
      while (nc < sc.n_cols && nc < 64) nc *= 2;
      variant = 500 + nc;
    } else if (sc.n_cols > 16 && sc.n_cols <= 32) {
      variant = 632;  // 17-32 FP64 columns: 32-B segments, one launch (3.50 vs 3.76 ms at 32 columns)
    } else {
      int nc = 2;
      while (nc < sc.n_cols && nc < 16) nc *= 2;
      variant = 300 + nc;
    }
  }
  const int family = variant / 100;  // 3/4: 16-B segment per lane, 5/6: 32-B segment
  const bool seq = family == 3 || family == 5;
  const bool wide = family >= 5;
  const int nc = variant % 100 + (variant % 100 == 28 ? 100 : 0);  // 528 / 628 = 128 columns
  if (family >= 3 && family <= 6) {
    if (precision == 64) {
      if (!wide) {
        switch (nc) {
          case 2: return launch_spmv<64, 2, 1>(md, sc, x, y, seq, stream);
          case 4: return launch_spmv<64, 4, 1>(md, sc, x, y, seq, stream);
          case 8: return launch_spmv<64, 8, 1>(md, sc, x, y, seq, stream);
          case 16: return launch_spmv<64, 16, 1>(md, sc, x, y, seq, stream);
          case 32: return launch_spmv<64, 32, 1>(md, sc, x, y, seq, stream);
          default: break;
        }
      } else {
        switch (nc) {
          case 4: return launch_spmv<64, 2, 2>(md, sc, x, y, seq, stream);
          case 8: return launch_spmv<64, 4, 2>(md, sc, x, y, seq, stream);
          case 16: return launch_spmv<64, 8, 2>(md, sc, x, y, seq, stream);
          case 32: return launch_spmv<64, 16, 2>(md, sc, x, y, seq, stream);
          case 64: return launch_spmv<64, 32, 2>(md, sc, x, y, seq, stream);
          default: break;
        }
      }
    } else {
      if (!wide) {
        switch (nc) {
          case 4: return launch_spmv<32, 2, 2>(md, sc, x, y, seq, stream);
          case 8: return launch_spmv<32, 4, 2>(md, sc, x, y, seq, stream);
          case 16: return launch_spmv<32, 8, 2>(md, sc, x, y, seq, stream);
          case 32: return launch_spmv<32, 16, 2>(md, sc, x, y, seq, stream);
          case 64: return launch_spmv<32, 32, 2>(md, sc, x, y, seq, stream);
          default: break;
        }
      } else {
        switch (nc) {
          case 8: return launch_spmv<32, 2, 4>(md, sc, x, y, seq, stream);
          case 16: return launch_spmv<32, 4, 4>(md, sc, x, y, seq, stream);
          case 32: return launch_spmv<32, 8, 4>(md, sc, x, y, seq, stream);
          case 64: return launch_spmv<32, 16, 4>(md, sc, x, y, seq, stream);
          case 128: return launch_spmv<32, 32, 4>(md, sc, x, y, seq, stream);
          default: break;
        }
      }
    }
  }
  return rsed_set_error(RSED_EINVAL, "projection apply variant %d invalid at precision %d", variant, precision);
}

extern "C" size_t rsed_proj_scratch_bytes(int64_t n_orbits) {
  return align_up(sizeof(int64_t) * (size_t)(n_orbits + 1), 256) + rsed_scan_scratch_bytes(n_orbits);
}

extern "C" int rsed_proj_count(const rsed_model_t* md, int64_t* rowptr, int64_t* n_hops_out, void* scratch,
                               size_t scratch_bytes, void* stream_) {
  int rc = check_proj_model(md);
  if (rc) return rc;
  RSED_REQUIRE(rowptr && n_hops_out && scratch, RSED_EINVAL, "bad projection count arguments");
  RSED_REQUIRE(scratch_bytes >= rsed_proj_scratch_bytes(md->n_orbits), RSED_ESCRATCH,
               "projection scratch too small");
  cudaStream_t stream = as_stream(stream_);
  int64_t* counts = reinterpret_cast<int64_t*>(scratch);
  char* scan = reinterpret_cast<char*>(scratch) + align_up(sizeof(int64_t) * (size_t)(md->n_orbits + 1), 256);
  rsed_sectors_t none{};
  ApplySmemLayout lay = apply_layout(*md, none);
  RSED_REQUIRE(lay.total <= 48 * 1024, RSED_ERANGE, "term tables exceed 48 KB of shared memory");
  k_proj_count<<<(unsigned)((md->n_orbits + 255) / 256), 256, lay.total, stream>>>(*md, counts, lay);
  RSED_CHECK_LAUNCH();
  rc = rsed_exclusive_scan_i64(counts, rowptr, md->n_orbits, scan, rsed_scan_scratch_bytes(md->n_orbits),
                               stream);
  if (rc) return rc;
  RSED_TRY_CUDA(cudaMemcpyAsync(n_hops_out, rowptr + md->n_orbits, sizeof(int64_t), cudaMemcpyDeviceToHost,
                                stream));
  RSED_TRY_CUDA(cudaStreamSynchronize(stream));
  return RSED_OK;
}

extern "C" int rsed_proj_fill(const rsed_model_t* md, const double* sqrt_stab, const int64_t* rowptr,
                              uint32_t* cg, double* w64, float* w32, void* stream_) {
  int rc = check_proj_model(md);
  if (rc) return rc;
  RSED_REQUIRE(sqrt_stab && rowptr && (cg || w64 || w32), RSED_EINVAL, "bad projection fill arguments");
  cudaStream_t stream = as_stream(stream_);
  rsed_sectors_t none{};
  ApplySmemLayout lay = apply_layout(*md, none);
  RSED_REQUIRE(lay.total <= 48 * 1024, RSED_ERANGE, "term tables exceed 48 KB of shared memory");
  k_proj_fill<4><<<(unsigned)((md->n_orbits + 255) / 256), 256, lay.total, stream>>>(
      *md, sqrt_stab, rowptr, cg, reinterpret_cast<double2*>(w64), reinterpret_cast<float2*>(w32), lay);
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}
