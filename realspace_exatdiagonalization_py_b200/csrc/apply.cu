// K6: matrix-free H|psi> over a block of columns (many sectors x block vectors)
// K7: matrix-mode triplets of one sector block, and a CSR SpMV.
//
// Vectors are row-major [n_orbits][ld]: row o is orbit o of the catalog, each
// column belongs to one momentum sector; rows of orbits outside a column's
// sector hold zero.  One hop gathers the 16-B table entry once and the whole
// contiguous row segment x[c][0..n_cols) once, so the table gather is shared
// by every sector and block vector of the batch.
#include <type_traits>
#include "rsed_internal.cuh"
#include "rsed_apply.cuh"

using namespace rsed_apply;

namespace {

template <typename XT>
struct XLoad;
template <>
struct XLoad<double2> {
  static __device__ __forceinline__ double2 ld(const double2* p) { return __ldg(p); }
};
template <>
struct XLoad<float2> {
  static __device__ __forceinline__ double2 ld(const float2* p) {
    float2 v = __ldg(p);
    return make_double2(v.x, v.y);
  }
};

// LPR lanes cooperate on one row; lane q owns columns q, q+LPR, ... (CPL of them).
// PREC 64: complex128 input and accumulation.  PREC 32: complex64 input and
// accumulation (the per-hop weight is formed in FP64 and rounded once).
// Hops are gathered HB at a time: all table entries of a batch are loaded
// together, then the member masks, sqrt|Stab| and x rows of their targets,
// so each batch costs two dependent memory round trips instead of 3*HB.
template <int LPR, int CPL, int PREC, int HB>
__global__ void __launch_bounds__(256) k_apply(rsed_model_t md, rsed_sectors_t sc, const void* xin,
                                               double2* __restrict__ y, ApplySmemLayout lay) {
  extern __shared__ __align__(16) unsigned char smem[];
  ApplyView v = stage_apply(md, sc, lay, smem);
  using XT = typename std::conditional<PREC == 64, double2, float2>::type;
  using AT = typename std::conditional<PREC == 64, double2, float2>::type;
  const XT* __restrict__ x = reinterpret_cast<const XT*>(xin);
  const int64_t gt = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t row = gt / LPR;
  const int q = (int)(gt % LPR);
  if (row >= md.n_orbits) return;
  const int kp1 = md.n_filled + 1;
  const int64_t cbs = md.species_b ? v.binom[__popcll(md.species_b) * kp1 + md.n_filled_b] : 1;
  const uint64_t m = md.repr_masks[row];
  const uint64_t memr = sc.member[row];
  int col[CPL], sec[CPL];
  bool on[CPL];
  AT acc[CPL];
  bool any = false;
#pragma unroll
  for (int j = 0; j < CPL; ++j) {
    col[j] = q + j * LPR;
    sec[j] = (col[j] < sc.n_cols) ? v.csec[col[j]] : 0;
    on[j] = (col[j] < sc.n_cols) && ((memr >> sec[j]) & 1ull);
    any |= on[j];
    acc[j].x = 0;
    acc[j].y = 0;
  }
  if (any) {
    const double2 hd = reinterpret_cast<const double2*>(md.hdiag)[row];
    const double sr = sc.sqrt_stab[row];
    // diagonal: conj(h) x[row]
#pragma unroll
    for (int j = 0; j < CPL; ++j) {
      if (!on[j]) continue;
      double2 xv = XLoad<XT>::ld(x + row * sc.ld + col[j]);
      double2 c = make_double2(hd.x * xv.x + hd.y * xv.y, hd.x * xv.y - hd.y * xv.x);
      acc[j].x += c.x;
      acc[j].y += c.y;
    }
    int bt[HB];
    int64_t bidx[HB];
    int nh = 0;
    auto process = [&](int cnt) {
      RsedEntry e[HB];
#pragma unroll
      for (int h = 0; h < HB; ++h)
        if (h < cnt) e[h] = load_entry(reinterpret_cast<const RsedEntry*>(md.table), bidx[h]);
      uint64_t mc[HB];
      double sq[HB];
      XT xv[HB][CPL];
#pragma unroll
      for (int h = 0; h < HB; ++h) {
        if (h < cnt) {
          const int64_t c = e[h].rep;
          mc[h] = __ldg(sc.member + c);
          sq[h] = __ldg(sc.sqrt_stab + c);
#pragma unroll
          for (int j = 0; j < CPL; ++j)
            if (on[j]) xv[h][j] = __ldg(x + c * sc.ld + col[j]);
        }
      }
#pragma unroll
      for (int h = 0; h < HB; ++h) {
        if (h >= cnt || (mc[h] & memr) == 0ull) continue;
        const int t = bt[h];
        // H[c, row] = t * s_JW * alpha * conj(chi(g)) * sqrt(S_c / S_row); we
        // accumulate its conjugate: w * chi(g) with w = conj(t s alpha) * ratio.
        double2 ta = cmul(v.tamp[t], make_double2(e[h].re, e[h].im));
        if (md.fermionic && (__popcll(m & v.tjw[t]) & 1)) {
          ta.x = -ta.x;
          ta.y = -ta.y;
        }
        const double ratio = sq[h] / sr;
        const double2 w = make_double2(ta.x * ratio, -ta.y * ratio);
#pragma unroll
        for (int j = 0; j < CPL; ++j) {
          if (!on[j] || !((mc[h] >> sec[j]) & 1ull)) continue;
          const double2 ch = v.chi[sec[j] * md.n_group + e[h].g];
          const double2 wc = cmul(w, ch);
          if constexpr (PREC == 64) {
            const double2 xx = xv[h][j];
            acc[j].x += wc.x * xx.x - wc.y * xx.y;
            acc[j].y += wc.x * xx.y + wc.y * xx.x;
          } else {
            const float2 xx = xv[h][j];
            const float2 wf = make_float2((float)wc.x, (float)wc.y);
            acc[j].x += wf.x * xx.x - wf.y * xx.y;
            acc[j].y += wf.x * xx.y + wf.y * xx.x;
          }
        }
      }
    };
    uint64_t occ = m;
    while (occ) {
      const int i = __ffsll((long long)occ) - 1;
      occ &= occ - 1;
      const int t1 = v.tbeg[i + 1];
      for (int t = v.tbeg[i]; t < t1; ++t) {
        const int jj = v.tto[t];
        if ((m >> jj) & 1ull) continue;
        bt[nh] = t;
        bidx[nh] = rsed_rank_any(m ^ (1ull << i) ^ (1ull << jj), v.binom, kp1, md.species_b, cbs);
        if (++nh == HB) {
          process(HB);
          nh = 0;
        }
      }
    }
    if (nh) process(nh);
  }
#pragma unroll
  for (int j = 0; j < CPL; ++j) {
    if (col[j] < sc.n_cols) {
      double2 o = on[j] ? make_double2((double)acc[j].x, (double)acc[j].y) : make_double2(0.0, 0.0);
      y[row * sc.ld + col[j]] = o;
    }
  }
}

template <int LPR, int CPL, int PREC, int HB = 4>
int launch_apply(const rsed_model_t& md, const rsed_sectors_t& sc, const void* x, double2* y,
                 cudaStream_t stream) {
  ApplySmemLayout lay = apply_layout(md, sc);
  if (lay.total > 48 * 1024) {
    RSED_TRY_CUDA(cudaFuncSetAttribute(k_apply<LPR, CPL, PREC, HB>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lay.total));
  }
  const int threads = 256;
  const int64_t total = md.n_orbits * LPR;
  const unsigned blocks = (unsigned)((total + threads - 1) / threads);
  k_apply<LPR, CPL, PREC, HB><<<blocks, threads, lay.total, stream>>>(md, sc, x, y, lay);
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}

template <int PREC>
int dispatch_apply(const rsed_model_t& md, const rsed_sectors_t& sc, const void* x, double2* y,
                   int variant, cudaStream_t stream) {
  const int n = sc.n_cols;
  // variant 0 = automatic choice by column count
  if (variant == 0) {
    if (n <= 1) variant = 1;
    else if (n <= 2) variant = 2;
    else if (n <= 4) variant = 3;
    else if (n <= 8) variant = 4;
    else if (n <= 16) variant = 5;
    else if (n <= 32) variant = 6;
    else if (n <= 64) variant = 7;
    else variant = 8;
  }
  switch (variant) {
    case 1: if (n <= 1) return launch_apply<1, 1, PREC>(md, sc, x, y, stream); break;
    case 2: if (n <= 2) return launch_apply<1, 2, PREC>(md, sc, x, y, stream); break;
    case 3: if (n <= 4) return launch_apply<1, 4, PREC>(md, sc, x, y, stream); break;
    case 4: if (n <= 8) return launch_apply<4, 2, PREC>(md, sc, x, y, stream); break;
    case 5: if (n <= 16) return launch_apply<8, 2, PREC>(md, sc, x, y, stream); break;
    case 6: if (n <= 32) return launch_apply<16, 2, PREC>(md, sc, x, y, stream); break;
    case 7: if (n <= 64) return launch_apply<32, 2, PREC>(md, sc, x, y, stream); break;
    case 8: if (n <= 128) return launch_apply<32, 4, PREC>(md, sc, x, y, stream); break;
    case 9: if (n <= 32) return launch_apply<32, 1, PREC>(md, sc, x, y, stream); break;
    case 10: if (n <= 16) return launch_apply<16, 1, PREC>(md, sc, x, y, stream); break;
    case 11: if (n <= 8) return launch_apply<8, 1, PREC>(md, sc, x, y, stream); break;
    case 12: if (n <= 4) return launch_apply<2, 2, PREC>(md, sc, x, y, stream); break;
    case 13: if (n <= 64) return launch_apply<16, 4, PREC>(md, sc, x, y, stream); break;
    // one hop at a time (no batching), for comparison
    case 101: if (n <= 1) return launch_apply<1, 1, PREC, 1>(md, sc, x, y, stream); break;
    case 106: if (n <= 32) return launch_apply<16, 2, PREC, 1>(md, sc, x, y, stream); break;
    case 107: if (n <= 64) return launch_apply<32, 2, PREC, 1>(md, sc, x, y, stream); break;
    // deeper hop batches
    case 201: if (n <= 1) return launch_apply<1, 1, PREC, 8>(md, sc, x, y, stream); break;
    case 206: if (n <= 32) return launch_apply<16, 2, PREC, 8>(md, sc, x, y, stream); break;
    case 207: if (n <= 64) return launch_apply<32, 2, PREC, 8>(md, sc, x, y, stream); break;
    case 209: if (n <= 32) return launch_apply<32, 1, PREC, 8>(md, sc, x, y, stream); break;
    default: break;
  }
  return rsed_set_error(RSED_EINVAL, "apply variant %d cannot hold %d columns", variant, n);
}

// ---- K7: exact triplets of one sector block ---------------------------------
// Column r of the block (orbit o = orbit_of_row[r]) produces, for every hop
// whose target lies in the sector, the entry (row = row_of_orbit[c], col = r)
// with value ((((t * s) * alpha) * conj(chi(g))) * sqrt(S_row / S_col)), the
// product order of symmetry_resolved_ed.py:686-687; the diagonal h_diag is a
// separate (r, r) entry first (include_diagonal, :648-651).
struct TripletCtx {
  rsed_model_t md;
  int64_t n_rows;
  const int32_t* orbit_of_row;
  const int32_t* row_of_orbit;
  const double2* chi;
  const double* sqrt_stab_unused;
};

__device__ __forceinline__ int stab_order_of(const uint64_t* stab_mask, int64_t o) {
  return __popcll(stab_mask[o]);
}

template <bool FILL>
__global__ void k_triplets(rsed_model_t md, int64_t n_rows, const int32_t* orbit_of_row,
                           const int32_t* row_of_orbit, const double2* chi, const uint64_t* stab_mask,
                           int64_t* col_count, const int64_t* col_off, int64_t* rows, int64_t* cols,
                           double2* vals, ApplySmemLayout lay) {
  extern __shared__ __align__(16) unsigned char smem[];
  // stage binomials and terms only
  int64_t* b = reinterpret_cast<int64_t*>(smem + lay.binom);
  int nb = (md.n_site + 1) * (md.n_filled + 1);
  for (int i = threadIdx.x; i < nb; i += blockDim.x) b[i] = md.binom[i];
  int32_t* tb = reinterpret_cast<int32_t*>(smem + lay.tbeg);
  for (int i = threadIdx.x; i <= md.n_site; i += blockDim.x) tb[i] = md.term_begin[i];
  uint8_t* tt = smem + lay.tto;
  double2* ta = reinterpret_cast<double2*>(smem + lay.tamp);
  uint64_t* tj = reinterpret_cast<uint64_t*>(smem + lay.tjw);
  for (int i = threadIdx.x; i < md.n_terms; i += blockDim.x) {
    tt[i] = md.term_to[i];
    ta[i] = reinterpret_cast<const double2*>(md.term_amp)[i];
    tj[i] = md.term_jw[i];
  }
  __syncthreads();
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_rows) return;
  const int kp1 = md.n_filled + 1;
  const int64_t cbs = md.species_b ? b[__popcll(md.species_b) * kp1 + md.n_filled_b] : 1;
  const int64_t o = orbit_of_row[r];
  const uint64_t m = md.repr_masks[o];
  const int s_col = stab_order_of(stab_mask, o);
  int64_t n = 1;  // diagonal entry
  int64_t pos = FILL ? col_off[r] : 0;
  if (FILL) {
    rows[pos] = r;
    cols[pos] = r;
    vals[pos] = reinterpret_cast<const double2*>(md.hdiag)[o];
    ++pos;
  }
  uint64_t occ = m;
  while (occ) {
    const int i = __ffsll((long long)occ) - 1;
    occ &= occ - 1;
    for (int t = tb[i]; t < tb[i + 1]; ++t) {
      const int jj = tt[t];
      if ((m >> jj) & 1ull) continue;
      const uint64_t m2 = m ^ (1ull << i) ^ (1ull << jj);
      const int64_t idx = rsed_rank_any(m2, b, kp1, md.species_b, cbs);
      const RsedEntry e = load_entry(reinterpret_cast<const RsedEntry*>(md.table), idx);
      const int32_t rr = row_of_orbit[e.rep];
      if (rr < 0) continue;
      if (FILL) {
        double2 hp = make_double2(1.0, 0.0);
        if (md.fermionic && (__popcll(m & tj[t]) & 1)) hp = make_double2(-1.0, 0.0);
        double2 v = cmul(ta[t], hp);
        v = cmul(v, make_double2((double)e.re, (double)e.im));
        double2 ch = chi[e.g];
        v = cmul(v, make_double2(ch.x, -ch.y));
        const int s_row = stab_order_of(stab_mask, e.rep);
        const double sq = sqrt((double)s_row / (double)s_col);
        v = cmul(v, make_double2(sq, 0.0));
        rows[pos] = rr;
        cols[pos] = r;
        vals[pos] = v;
        ++pos;
      }
      ++n;
    }
  }
  if (!FILL) col_count[r] = n;
}

__global__ void k_csr_spmv(int64_t n_rows, const int64_t* rp, const int32_t* ci, const double2* va,
                           int n_vec, const double2* x, double2* y) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_rows) return;
  for (int v = 0; v < n_vec; ++v) {
    double2 acc = make_double2(0.0, 0.0);
    for (int64_t p = rp[r]; p < rp[r + 1]; ++p) {
      const double2 a = va[p];
      const double2 b = x[(int64_t)v * n_rows + ci[p]];
      acc.x += a.x * b.x - a.y * b.y;
      acc.y += a.x * b.y + a.y * b.x;
    }
    y[(int64_t)v * n_rows + r] = acc;
  }
}

}  // namespace

static int check_model(const rsed_model_t* md) {
  RSED_REQUIRE(md != nullptr, RSED_EINVAL, "model descriptor is NULL");
  RSED_REQUIRE(md->n_site >= 1 && md->n_site <= RSED_MAX_SITES, RSED_ERANGE, "bad n_site");
  RSED_REQUIRE(md->n_group >= 1 && md->n_group <= RSED_MAX_GROUP, RSED_ERANGE, "bad |G|");
  RSED_REQUIRE(md->n_orbits >= 1 && md->table && md->repr_masks && md->binom && md->hdiag,
               RSED_EINVAL, "model tables missing");
  RSED_REQUIRE(md->n_terms >= 0 && md->term_begin, RSED_EINVAL, "terms missing");
  RSED_REQUIRE(md->n_terms == 0 || (md->term_to && md->term_amp && md->term_jw), RSED_EINVAL,
               "terms missing");
  return RSED_OK;
}

extern "C" int rsed_apply_h(const rsed_model_t* md, const rsed_sectors_t* sc, const void* x, void* y,
                            int32_t precision, int32_t variant, void* stream_) {
  int rc = check_model(md);
  if (rc) return rc;
  RSED_REQUIRE(sc && sc->member && sc->sqrt_stab && sc->chi && sc->col_sector, RSED_EINVAL,
               "sector descriptor incomplete");
  RSED_REQUIRE(sc->n_cols >= 1 && sc->ld >= sc->n_cols && sc->n_sectors >= 1 && sc->n_sectors <= 64,
               RSED_EINVAL, "bad column layout");
  RSED_REQUIRE(sc->n_group == md->n_group, RSED_EINVAL, "sector/model group order mismatch");
  RSED_REQUIRE(x && y, RSED_EINVAL, "x or y is NULL");
  cudaStream_t stream = as_stream(stream_);
  RSED_REQUIRE(precision == 64 || precision == 32, RSED_EINVAL, "precision must be 64 or 32");
  const bool have_proj =
      md->proj_rowptr && md->proj_cg && (precision == 64 ? md->proj_w64 != nullptr : md->proj_w32 != nullptr);
  if (variant == 999) {
    variant = 0;  // automatic on-the-fly mapping even when a projection table is present
  } else if (variant >= 300 || (variant == 0 && have_proj)) {
    return rsed_proj_apply(*md, *sc, x, reinterpret_cast<double2*>(y), precision, variant, stream);
  }
  if (precision == 64)
    return dispatch_apply<64>(*md, *sc, x, reinterpret_cast<double2*>(y), variant, stream);
  if (precision == 32)
    return dispatch_apply<32>(*md, *sc, x, reinterpret_cast<double2*>(y), variant, stream);
  return rsed_set_error(RSED_EINVAL, "precision must be 64 or 32");
}

extern "C" size_t rsed_triplet_scratch_bytes(int64_t n_rows) {
  return align_up(sizeof(int64_t) * (size_t)(n_rows + 1), 256) + rsed_scan_scratch_bytes(n_rows);
}

static ApplySmemLayout triplet_layout(const rsed_model_t* md) {
  rsed_sectors_t sc{};
  sc.n_sectors = 0;
  sc.n_cols = 0;
  return apply_layout(*md, sc);
}

extern "C" int rsed_triplets_count(const rsed_model_t* md, int64_t n_rows, const int32_t* orbit_of_row,
                                   const int32_t* row_of_orbit, const double* chi,
                                   const uint64_t* stab_mask, int64_t* col_off, int64_t* nnz_out,
                                   void* scratch, size_t scratch_bytes, void* stream_) {
  int rc = check_model(md);
  if (rc) return rc;
  RSED_REQUIRE(n_rows >= 1 && orbit_of_row && row_of_orbit && chi && stab_mask && col_off && nnz_out,
               RSED_EINVAL, "bad triplet arguments");
  RSED_REQUIRE(scratch_bytes >= rsed_triplet_scratch_bytes(n_rows), RSED_ESCRATCH,
               "triplet scratch too small");
  cudaStream_t stream = as_stream(stream_);
  int64_t* counts = reinterpret_cast<int64_t*>(scratch);
  char* scan = reinterpret_cast<char*>(scratch) + align_up(sizeof(int64_t) * (size_t)(n_rows + 1), 256);
  ApplySmemLayout lay = triplet_layout(md);
  k_triplets<false><<<(unsigned)((n_rows + 127) / 128), 128, lay.total, stream>>>(
      *md, n_rows, orbit_of_row, row_of_orbit, reinterpret_cast<const double2*>(chi), stab_mask,
      counts, nullptr, nullptr, nullptr, nullptr, lay);
  RSED_CHECK_LAUNCH();
  rc = rsed_exclusive_scan_i64(counts, col_off, n_rows, scan, rsed_scan_scratch_bytes(n_rows), stream);
  if (rc) return rc;
  RSED_TRY_CUDA(cudaMemcpyAsync(nnz_out, col_off + n_rows, sizeof(int64_t), cudaMemcpyDeviceToHost,
                                stream));
  RSED_TRY_CUDA(cudaStreamSynchronize(stream));
  return RSED_OK;
}

extern "C" int rsed_triplets_fill(const rsed_model_t* md, int64_t n_rows, const int32_t* orbit_of_row,
                                  const int32_t* row_of_orbit, const double* chi,
                                  const uint64_t* stab_mask, const int64_t* col_off, int64_t* rows,
                                  int64_t* cols, double* vals, void* stream_) {
  int rc = check_model(md);
  if (rc) return rc;
  RSED_REQUIRE(n_rows >= 1 && orbit_of_row && row_of_orbit && chi && stab_mask && col_off && rows &&
                   cols && vals,
               RSED_EINVAL, "bad triplet arguments");
  cudaStream_t stream = as_stream(stream_);
  ApplySmemLayout lay = triplet_layout(md);
  k_triplets<true><<<(unsigned)((n_rows + 127) / 128), 128, lay.total, stream>>>(
      *md, n_rows, orbit_of_row, row_of_orbit, reinterpret_cast<const double2*>(chi), stab_mask,
      nullptr, col_off, rows, cols, reinterpret_cast<double2*>(vals), lay);
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}

extern "C" int rsed_csr_spmv(int64_t n_rows, const int64_t* row_ptr, const int32_t* col_idx,
                             const double* vals, int32_t n_vec, const double* x, double* y,
                             void* stream_) {
  RSED_REQUIRE(n_rows >= 1 && row_ptr && col_idx && vals && x && y && n_vec >= 1, RSED_EINVAL,
               "bad CSR arguments");
  cudaStream_t stream = as_stream(stream_);
  k_csr_spmv<<<(unsigned)((n_rows + 255) / 256), 256, 0, stream>>>(
      n_rows, row_ptr, col_idx, reinterpret_cast<const double2*>(vals), n_vec,
      reinterpret_cast<const double2*>(x), reinterpret_cast<double2*>(y));
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}
