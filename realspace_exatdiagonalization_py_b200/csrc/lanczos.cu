// K8: batched thick-restart block Lanczos with full FP64 reorthogonalisation.
//
// One batch holds n_inst independent eigen-solves ("instances", e.g. the
// momentum sectors of one lattice/flux point).  Instance i owns b_i columns
// [c0_i, c0_i + b_i) of every block buffer; all blocks share the row-major
// [n_orbits][ld] layout of the matrix-free apply, so one apply launch serves
// every instance.  Per iteration (all kernels launched unconditionally, each
// instance decides from its device-side state whether it has work, so a
// sequence of iterations can be captured in one CUDA graph):
//
//   apply    W = H X                      (X = newest basis block)
//   pass 1   C1 = V^H W, G1 = W^H W  ->  R1 = chol(G1 - C1^H C1),  W = (W - V C1) R1^-1
//   pass 2   C2, G2 on the new W     ->  R2,  V_new = (W - V C2) R2^-1
//            P[:, cur] = C1 + C2 R1,  P[new, cur] = R2 R1   (projected matrix)
//   ritz     (some iterations) Jacobi eigen-solve of (P + P^H)/2 in shared
//            memory, residual estimates |R_last S_last,j|, convergence test,
//            thick restart bookkeeping
//   restart  V_0..keep-1 = V S_keep, residual block moved behind them
//
// The reorthogonalisation is block classical Gram-Schmidt with the Pythagorean
// Cholesky update, one reduction per pass.  With the adaptive single pass
// (st.reserved bit 0), pass 1 orthogonalises W_loc = W - sigma X - sum_{l<j}
// V_l P[j, l]^H, i.e. W with the part of the Lanczos recurrence already known
// from the projected matrix removed (the coupling to the previous block, or
// to the Ritz vectors after a thick restart, and a shift sigma = diag of the
// previous diagonal block), formed row by row while W is staged; when the
// smallest Cholesky pivot of W_loc - V C still carries at least 1/8 of its
// column's squared norm (little cancellation: orthogonality and
// normalisation after one pass are within a few ulps of two passes), pass 1
// writes the new basis block directly and pass 2 is skipped for that
// instance; otherwise pass 2 runs as before.
#include <cooperative_groups.h>
#include <type_traits>
#include "rsed_internal.cuh"
#include "rsed_apply.cuh"

namespace cg = cooperative_groups;

extern "C" int64_t rsed_lanczos_partial_len(int64_t n_orbits, int32_t chunk_rows, int32_t n_inst,
                                            int32_t n_slots);

namespace {

constexpr int kBMax = 8;        // largest block per instance
constexpr int kKeepMax = 16;    // largest thick-restart basis (columns)
constexpr int kJacobiMax = 64;  // largest projected matrix
constexpr int kRRMax = kKeepMax + kBMax;  // Rayleigh-Ritz basis (restart basis + residual block)
constexpr int kStateInts = 16;
// the eigensolver's shared work area for the inverse iteration: five double
// arrays and the pivot flags of kKeepMax vectors of up to kJacobiMax entries
constexpr size_t kHermWork = sizeof(double) * 5 * kJacobiMax * kKeepMax + kJacobiMax * kKeepMax;
// dynamic shared memory of k_lz_ritz: padded A (M x (M+1)), S (M x 16 complex), Z (M x 16 real),
// then the eigensolver's work area
constexpr size_t kRitzSmem = sizeof(double2) * (kJacobiMax * (kJacobiMax + 1) + kJacobiMax * kKeepMax) +
                             sizeof(double) * kJacobiMax * kKeepMax + kHermWork;
// state fields
constexpr int S_NB = 0, S_STATUS = 1, S_RESTARTS = 2, S_ITERS = 3, S_ACTIVE = 4, S_RESTART_NB = 5,
              S_NEWSLOT = 6, S_NCONV = 7, S_TICKET = 8, S_RR = 9, S_ONEPASS = 10, S_ONEPASS_N = 11,
              S_RED_BLOCKS = 12, S_PASSES = 13;  // basis blocks + W read by the executed passes, passes
// single pass allowed when every Cholesky pivot^2 >= G_qq / kOnePassKappa2
constexpr double kOnePassKappa2 = 8.0;
constexpr int kFlagSinglePass = 1;

struct LzDims {
  int64_t n_orb;
  int ld;
  int n_inst;
  int n_slots;
  int pm;
  int chunk_rows;
  int n_chunks;
  int pslots;  // n_slots + 2 reduction slots per instance
};

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
// conj(a) * b
__device__ __forceinline__ double2 cdotc(double2 a, double2 b) {
  return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

// ---------------------------------------------------------------------------
// Reduction + finalisation in one launch.  Block (chunk, inst) forms
//   partial[chunk][inst][s][p][q] = sum_rows conj(Y_s[row][c0+p]) W[row][c0+q]
// with Y_s = V[s] for s < nb and Y_nb = W (Gram of W itself); the last block
// of an instance to finish (atomic ticket, no waiting) sums the partials in
// chunk order, forms G' = G - C^H C, its Cholesky factor R and the
// projected-matrix entries.
constexpr int kRT = 256;         // threads of k_lz_reduce
constexpr int kTileRows = 256;  // rows of W staged in shared memory per tile

// This chunk's Gram partials for one instance with block size BB: warp w owns
// slots w, w+8, w+16, ... (slot nb = W itself) and keeps their sums in
// registers across all row tiles; W's rows are staged tile by tile in shared
// memory, so V and W are each read once, as whole row segments.  Lane sums
// are combined in shared memory in a fixed order.
template <int BB>
__device__ void lz_gram_chunk(const double2* __restrict__ V, const double2* __restrict__ W, int64_t slot_stride,
                              int64_t ld, int c0, int nb, int64_t r0, int64_t r1, double2* __restrict__ out,
                              double2* buf, const double2* Lc, const int* lnz, const double* sig, int jloc) {
  constexpr int SW = (kJacobiMax / BB + 1 + 7) / 8;  // most slots one warp owns
  constexpr int RPW = 32 / BB;                       // rows per warp pass
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int rl = lane / BB, p = lane % BB;
  const bool act = rl < RPW;
  double2 acc[SW][BB];
#pragma unroll
  for (int j = 0; j < SW; ++j)
#pragma unroll
    for (int q = 0; q < BB; ++q) acc[j][q] = make_double2(0.0, 0.0);
  double2* Wt = buf;  // [kTileRows][BB]
  for (int64_t t0 = r0; t0 < r1; t0 += kTileRows) {
    const int nr = (int)min((int64_t)kTileRows, r1 - t0);
    __syncthreads();
    for (int i = threadIdx.x; i < nr * BB; i += kRT) {
      const int rr = i / BB, q = i % BB;
      const int64_t row = t0 + rr;
      double2 w = W[row * ld + c0 + q];
      if (jloc > 0) {
        // W_loc = W - sigma_q X_q - sum over the known couplings P[j, l]^H
        const double2 x = V[(int64_t)jloc * slot_stride + row * ld + c0 + q];
        w.x -= sig[q] * x.x;
        w.y -= sig[q] * x.y;
        for (int l = 0; l < jloc; ++l) {
          if (!lnz[l]) continue;
          const double2* Vl = V + (int64_t)l * slot_stride + row * ld + c0;
#pragma unroll
          for (int pp = 0; pp < BB; ++pp) w = csub(w, cmul(Vl[pp], Lc[(l * BB + pp) * kBMax + q]));
        }
      }
      Wt[rr * BB + q] = w;
    }
    __syncthreads();
    if (act) {
#pragma unroll
      for (int j = 0; j < SW; ++j) {
        const int sl = warp + 8 * j;
        if (sl > nb) break;
        if (sl < nb) {
          const double2* Y = V + sl * slot_stride + c0 + p;
#pragma unroll 4
          for (int rr = rl; rr < nr; rr += RPW) {
            const double2 y = Y[(t0 + rr) * ld];
#pragma unroll
            for (int q = 0; q < BB; ++q) acc[j][q] = cadd(acc[j][q], cdotc(y, Wt[rr * BB + q]));
          }
        } else {
          for (int rr = rl; rr < nr; rr += RPW) {
            const double2 y = Wt[rr * BB + p];
#pragma unroll
            for (int q = 0; q < BB; ++q) acc[j][q] = cadd(acc[j][q], cdotc(y, Wt[rr * BB + q]));
          }
        }
      }
    }
  }
  __syncthreads();
  double2(*red)[32][kBMax] = reinterpret_cast<double2(*)[32][kBMax]>(buf);  // reuses the tile
#pragma unroll
  for (int j = 0; j < SW; ++j) {
    const int sl = warp + 8 * j;
    if (sl > nb) break;
    if (act) {
#pragma unroll
      for (int q = 0; q < BB; ++q) red[warp][lane][q] = acc[j][q];
    }
    __syncwarp();
    if (lane < BB) {
#pragma unroll
      for (int q = 0; q < BB; ++q) {
        double2 t = make_double2(0.0, 0.0);
        for (int k = 0; k < RPW; ++k) t = cadd(t, red[warp][k * BB + lane][q]);
        out[sl * kBMax * kBMax + lane * kBMax + q] = t;
      }
    }
    __syncwarp();
  }
}

// Finalisation of one instance's Gram partials (one block of kRT threads):
// sum the chunk partials (G threads per entry over interleaved chunk subsets,
// then in order: deterministic for a given chunk count), form
// G' = G - C^H C, its Cholesky factor R and the projected-matrix entries.
__device__ void lz_finalize(const rsed_lanczos_t& st, const LzDims& d, int inst, int pass, int b, int nb, int* stt,
                            double2* sc, double2* sR, double2* sG, int* s_ok, double2* fin, bool loc,
                            int* s_one) {
  const double2* part = reinterpret_cast<const double2*>(st.partial);
  // ---- finalisation (one block per instance) ----
  // G threads per entry sum interleaved chunk subsets, then the G partial
  // sums are added in order (deterministic for a given chunk count)
  const int nent = (nb + 1) * b * b;
  const int G = max(1, kRT / nent);
  {
    // fin: kRT * kBMax >= nent * G entries
    const int64_t cstride = (int64_t)d.n_inst * d.pslots * kBMax * kBMax;
    for (int t = threadIdx.x; t < nent * G; t += kRT) {
      const int e = t % nent, g = t / nent;
      const int sl = e / (b * b), pq = e % (b * b), p = pq / b, q = pq % b;
      const double2* src = part + (int64_t)inst * d.pslots * kBMax * kBMax + sl * kBMax * kBMax + p * kBMax + q;
      double2 a = make_double2(0.0, 0.0);
#pragma unroll 8
      for (int c = g; c < d.n_chunks; c += G) a = cadd(a, __ldcg(src + c * cstride));
      fin[g * nent + e] = a;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nent; e += kRT) {
      const int sl = e / (b * b), pq = e % (b * b), p = pq / b, q = pq % b;
      double2 a = make_double2(0.0, 0.0);
      for (int g = 0; g < G; ++g) a = cadd(a, fin[g * nent + e]);
      sc[(sl * b + p) * kBMax + q] = a;  // row (sl*b + p), column q
    }
  }
  __syncthreads();
  // G' = G - C^H C, one thread per (p, q)
  for (int e = threadIdx.x; e < b * b; e += blockDim.x) {
    const int p = e / b, q = e % b;
    double2 g = sc[(nb * b + p) * kBMax + q];
    for (int r = 0; r < nb * b; ++r) g = csub(g, cdotc(sc[r * kBMax + p], sc[r * kBMax + q]));
    sG[p * kBMax + q] = g;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double gmax = 0.0;
    for (int p = 0; p < b; ++p) gmax = fmax(gmax, sc[(nb * b + p) * kBMax + p].x);
    for (int i = 0; i < kBMax * kBMax; ++i) sR[i] = make_double2(0.0, 0.0);
    bool ok = gmax > 0.0;
    for (int j = 0; j < b && ok; ++j) {
      double sdiag = sG[j * kBMax + j].x;
      for (int k = 0; k < j; ++k) sdiag -= sR[k * kBMax + j].x * sR[k * kBMax + j].x + sR[k * kBMax + j].y * sR[k * kBMax + j].y;
      if (!(sdiag > 1e-26 * gmax)) {
        ok = false;
        break;
      }
      const double rjj = sqrt(sdiag);
      sR[j * kBMax + j] = make_double2(rjj, 0.0);
      for (int q = j + 1; q < b; ++q) {
        double2 t = sG[j * kBMax + q];
        for (int k = 0; k < j; ++k) t = csub(t, cdotc(sR[k * kBMax + j], sR[k * kBMax + q]));
        sR[j * kBMax + q] = make_double2(t.x / rjj, t.y / rjj);
      }
    }
    *s_ok = ok;
    if (!ok) {
      stt[S_STATUS] = RSED_EBREAKDOWN;
      stt[S_ACTIVE] = 0;
    }
    // single pass when no pivot lost more than 7/8 of its column's norm^2
    bool one = ok && pass == 1 && nb >= 1 && (st.reserved & kFlagSinglePass);
    for (int q = 0; q < b && one; ++q) {
      const double gq = sc[(nb * b + q) * kBMax + q].x;
      one = sR[q * kBMax + q].x * sR[q * kBMax + q].x * kOnePassKappa2 >= gq;
    }
    *s_one = one;
    if (pass == 1) stt[S_ONEPASS] = one;
    if (ok) {
      stt[S_RED_BLOCKS] += nb + 1;
      stt[S_PASSES] += 1;
    }
  }
  __syncthreads();
  if (!*s_ok) return;
  if (loc) {
    // coefficients of W itself: C + the local part taken off before the Gram
    const double2* Pi = reinterpret_cast<const double2*>(st.P) + (int64_t)inst * d.pm * d.pm;
    const int j = nb - 1;
    for (int e = threadIdx.x; e < nb * b * b; e += blockDim.x) {
      const int r = e / b, q = e % b;
      double2 add;
      if (r < j * b) {
        add = cconj(Pi[(int64_t)(j * b + q) * d.pm + r]);
      } else {
        const int p = r - j * b;
        add = make_double2(p == q ? Pi[(int64_t)((j - 1) * b + q) * d.pm + (j - 1) * b + q].x : 0.0, 0.0);
      }
      sc[r * kBMax + q] = cadd(sc[r * kBMax + q], add);
    }
    __syncthreads();
  }
  double2* coefp = reinterpret_cast<double2*>(st.coef) + (int64_t)inst * 2 * d.pslots * kBMax * kBMax;
  double2* cp = coefp + (pass - 1) * d.pslots * kBMax * kBMax;
  for (int e = threadIdx.x; e < nb * b * b; e += blockDim.x) {
    const int r = e / b, q = e % b;  // C[s r'][q] stored slot-major as before
    cp[(r / b) * kBMax * kBMax + (r % b) * kBMax + q] = sc[r * kBMax + q];
  }
  double2* Rout = cp + (d.pslots - 1) * kBMax * kBMax;
  for (int e = threadIdx.x; e < kBMax * kBMax; e += blockDim.x) Rout[e] = sR[e];
  if (pass == 1 && *s_one) {
    // one pass: P[:, cur] = C1, P[new, cur] = R1
    double2* P = reinterpret_cast<double2*>(st.P) + (int64_t)inst * d.pm * d.pm;
    const int cb = nb - 1;
    for (int e = threadIdx.x; e < nb * b * b; e += blockDim.x) {
      const int r = e / b, q = e % b;
      P[(int64_t)r * d.pm + cb * b + q] = sc[r * kBMax + q];
    }
    for (int e = threadIdx.x; e < b * b; e += blockDim.x) {
      const int p = e / b, q = e % b;
      P[(int64_t)(nb * b + p) * d.pm + cb * b + q] = sR[p * kBMax + q];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      stt[S_NEWSLOT] = nb;
      stt[S_NB] = nb + 1;
      stt[S_ITERS] += 1;
      stt[S_ONEPASS_N] += 1;
    }
    return;
  }
  if (pass == 2) {
    const int nb_old = nb;
    if (nb_old >= 1) {
      // combine passes: C = C1 + C2 R1, Rtot = R2 R1 ; column block cb = nb_old-1
      const double2* c1 = coefp;
      const double2* R1 = coefp + (d.pslots - 1) * kBMax * kBMax;
      double2* P = reinterpret_cast<double2*>(st.P) + (int64_t)inst * d.pm * d.pm;
      const int cb = nb_old - 1;
      for (int e = threadIdx.x; e < nb_old * b * b; e += blockDim.x) {
        const int r = e / b, q = e % b, sl = r / b, p = r % b;
        double2 v = c1[sl * kBMax * kBMax + p * kBMax + q];
        for (int k = 0; k < b; ++k) v = cadd(v, cmul(sc[r * kBMax + k], R1[k * kBMax + q]));
        P[(int64_t)r * d.pm + cb * b + q] = v;
      }
      for (int e = threadIdx.x; e < b * b; e += blockDim.x) {
        const int p = e / b, q = e % b;
        double2 v = make_double2(0.0, 0.0);
        for (int k = 0; k < b; ++k) v = cadd(v, cmul(sR[p * kBMax + k], R1[k * kBMax + q]));
        P[(int64_t)(nb_old * b + p) * d.pm + cb * b + q] = v;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      stt[S_NEWSLOT] = nb_old;
      stt[S_NB] = nb_old + 1;
      stt[S_ITERS] += 1;
    }
  }
}

__global__ void __launch_bounds__(kRT) k_lz_reduce(rsed_lanczos_t st, LzDims d, int pass) {
  // blocks of all instances over one row chunk are adjacent in launch order:
  // they read the same rows (each its own columns), so L2 serves the rest of
  // every DRAM line one of them fetched
  const int chunk = blockIdx.x / d.n_inst;
  const int inst = blockIdx.x % d.n_inst;
  int* stt = st.state + inst * kStateInts;
  if (pass == 1 && chunk == 0 && threadIdx.x == 0) stt[S_RESTART_NB] = 0;
  if (!stt[S_ACTIVE]) return;
  if (pass == 2 && stt[S_ONEPASS]) return;  // pass 1 already wrote the new block
  const int b = st.inst_b[inst];
  const int c0 = st.inst_col0[inst];
  const int nb = stt[S_NB];
  __shared__ int s_last, s_one;
  __shared__ double s_sig[kBMax];
  __shared__ int s_lnz[kJacobiMax];
  __shared__ double2 sc[(kJacobiMax / 1 + kBMax + kBMax) * kBMax];  // C (nb*b rows) + G rows
  __shared__ double2 sR[kBMax * kBMax];
  __shared__ double2 sG[kBMax * kBMax];
  __shared__ int s_ok;
  if (nb > d.n_slots || b < 1 || b > kBMax || nb * b > kJacobiMax + kBMax) {
    // the basis is full (no restart happened) or the block size is invalid:
    // stop this instance instead of writing past its slots
    if (chunk == 0 && threadIdx.x == 0) {
      stt[S_STATUS] = RSED_EINVAL;
      stt[S_ACTIVE] = 0;
    }
    return;
  }
  const int64_t r0 = (int64_t)chunk * d.chunk_rows;
  const int64_t r1 = min(r0 + d.chunk_rows, d.n_orb);
  const double2* V = reinterpret_cast<const double2*>(st.V);
  const double2* W = reinterpret_cast<const double2*>(st.W);
  double2* part = reinterpret_cast<double2*>(st.partial);
  const int64_t slot_stride = d.n_orb * d.ld;
  const int64_t pbase = ((int64_t)chunk * d.n_inst + inst) * (int64_t)d.pslots * kBMax * kBMax;
  __shared__ double2 red_l[kRT / 32][32][kBMax];  // W tile, lane sums, then the finalisation's partials
  // the known part of the recurrence (pass 1 of a single-pass-enabled batch,
  // basis of two or more blocks): L[l*b + p][q] = conj(P[j*b + q][l*b + p])
  // for l < j = nb - 1 (staged in sc, which the finalisation rebuilds), and
  // sigma_q = Re P[(j-1)*b + q][(j-1)*b + q]
  const bool loc = pass == 1 && nb >= 2 && (st.reserved & kFlagSinglePass);
  const int jloc = loc ? nb - 1 : 0;
  if (loc) {
    const double2* Pi = reinterpret_cast<const double2*>(st.P) + (int64_t)inst * d.pm * d.pm;
    for (int e = threadIdx.x; e < jloc * b * b; e += kRT) {
      const int r = e / b, q = e % b;
      sc[r * kBMax + q] = cconj(Pi[(int64_t)(jloc * b + q) * d.pm + r]);
    }
    if (threadIdx.x < b)
      s_sig[threadIdx.x] = Pi[(int64_t)((jloc - 1) * b + threadIdx.x) * d.pm + (jloc - 1) * b + threadIdx.x].x;
    __syncthreads();
    for (int l = threadIdx.x; l < jloc; l += kRT) {
      int nz = 0;
      for (int e = 0; e < b * b; ++e) {
        const double2 v = sc[(l * b + e / b) * kBMax + e % b];
        nz |= (v.x != 0.0) || (v.y != 0.0);
      }
      s_lnz[l] = nz;
    }
    __syncthreads();
  }
  {
    double2* buf = &red_l[0][0][0];
    double2* out = part + pbase;
    switch (b) {
      case 1: lz_gram_chunk<1>(V, W, slot_stride, d.ld, c0, nb, r0, r1, out, buf, sc, s_lnz, s_sig, jloc); break;
      case 2: lz_gram_chunk<2>(V, W, slot_stride, d.ld, c0, nb, r0, r1, out, buf, sc, s_lnz, s_sig, jloc); break;
      case 3: lz_gram_chunk<3>(V, W, slot_stride, d.ld, c0, nb, r0, r1, out, buf, sc, s_lnz, s_sig, jloc); break;
      case 4: lz_gram_chunk<4>(V, W, slot_stride, d.ld, c0, nb, r0, r1, out, buf, sc, s_lnz, s_sig, jloc); break;
      case 5: lz_gram_chunk<5>(V, W, slot_stride, d.ld, c0, nb, r0, r1, out, buf, sc, s_lnz, s_sig, jloc); break;
      case 6: lz_gram_chunk<6>(V, W, slot_stride, d.ld, c0, nb, r0, r1, out, buf, sc, s_lnz, s_sig, jloc); break;
      case 7: lz_gram_chunk<7>(V, W, slot_stride, d.ld, c0, nb, r0, r1, out, buf, sc, s_lnz, s_sig, jloc); break;
      default: lz_gram_chunk<8>(V, W, slot_stride, d.ld, c0, nb, r0, r1, out, buf, sc, s_lnz, s_sig, jloc); break;
    }
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const int t = atomicAdd(&stt[S_TICKET], 1);
    s_last = (t == d.n_chunks - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (threadIdx.x == 0) stt[S_TICKET] = 0;
  __syncthreads();  // sc (local coefficients) is rebuilt by the finalisation
  lz_finalize(st, d, inst, pass, b, nb, stt, sc, sR, sG, &s_ok, &red_l[0][0][0], loc, &s_one);
}

// W <- (W - V C) R^-1 ; pass 2 writes the new basis block and the matvec input.
// Block (row range, instance), the instance's coefficients staged in shared
// memory; one thread per (row, column q) -- the b lanes of a row read the
// row's segment together and solve with R across lanes by shuffles.
__global__ void __launch_bounds__(256) k_lz_update(rsed_lanczos_t st, LzDims d, int pass) {
  const int inst = blockIdx.x % d.n_inst;  // instances of one row group adjacent in launch order
  const int64_t rgroup = blockIdx.x / d.n_inst;
  const int* stt = st.state + inst * kStateInts;
  if (!stt[S_ACTIVE]) return;
  const bool one = stt[S_ONEPASS] != 0;  // pass 1 writes the new block, pass 2 is skipped
  if (pass == 2 && one) return;
  const int b = st.inst_b[inst];
  const int c0 = st.inst_col0[inst];
  const int nb = (pass == 2 || one) ? stt[S_NEWSLOT] : stt[S_NB];
  if (nb * b > kJacobiMax || b > kBMax) return;  // guarded by k_lz_reduce (status set there)
  const double2* coef = reinterpret_cast<const double2*>(st.coef) +
                        (int64_t)inst * 2 * d.pslots * kBMax * kBMax + (pass - 1) * d.pslots * kBMax * kBMax;
  __shared__ double2 cs[kJacobiMax * kBMax];
  __shared__ double2 Rs[kBMax * kBMax];
  for (int e = threadIdx.x; e < nb * b * b; e += blockDim.x) {
    const int r = e / b, q = e % b;  // r = s * b + p
    cs[r * kBMax + q] = coef[(r / b) * kBMax * kBMax + (r % b) * kBMax + q];
  }
  for (int e = threadIdx.x; e < kBMax * kBMax; e += blockDim.x) Rs[e] = coef[(d.pslots - 1) * kBMax * kBMax + e];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int rpw = 32 / b;
  const int rl = lane / b, q = lane % b;
  const int64_t row = (rgroup * (blockDim.x >> 5) + warp) * rpw + rl;
  const bool act = rl < rpw && row < d.n_orb;
  double2* V = reinterpret_cast<double2*>(st.V);
  double2* W = reinterpret_cast<double2*>(st.W);
  const int64_t slot_stride = d.n_orb * d.ld;
  double2 w = make_double2(0.0, 0.0);
  if (act) {
    w = W[row * d.ld + c0 + q];
#pragma unroll 4
    for (int s = 0; s < nb; ++s) {
      const double2* Vs = V + s * slot_stride + row * d.ld + c0;
      for (int p = 0; p < b; ++p) w = csub(w, cmul(Vs[p], cs[(s * b + p) * kBMax + q]));
    }
  }
  // x R = w: x_q = (w_q - sum_{p<q} x_p R[p][q]) / R[q][q], across the row's lanes
  const int base = lane - q;
  double2 acc = make_double2(0.0, 0.0), xq = make_double2(0.0, 0.0);
  for (int pp = 0; pp < b; ++pp) {
    if (q == pp) {
      const double rr = Rs[pp * kBMax + pp].x;
      xq = make_double2((w.x - acc.x) / rr, (w.y - acc.y) / rr);
    }
    const int src = min(base + pp, 31);
    const double xpx = __shfl_sync(0xffffffffu, xq.x, src);
    const double xpy = __shfl_sync(0xffffffffu, xq.y, src);
    if (q > pp) acc = cadd(acc, cmul(make_double2(xpx, xpy), Rs[pp * kBMax + q]));
  }
  if (!act) return;
  if (pass == 1 && !one) {
    W[row * d.ld + c0 + q] = xq;
  } else {
    V[(int64_t)nb * slot_stride + row * d.ld + c0 + q] = xq;
    if (st.Xf == nullptr) V[(int64_t)(d.n_slots + 1) * slot_stride + row * d.ld + c0 + q] = xq;
    if (st.Xf) reinterpret_cast<float2*>(st.Xf)[row * d.ld + c0 + q] = make_float2((float)xq.x, (float)xq.y);
  }
}

// The same update for all instances at once (batches of 2+ instances whose
// coefficients fit in shared memory): a block holds every instance's
// coefficients and walks RG row groups at a time (thread = one column of one
// row in each group), so each slot is read as contiguous rows and every thread
// keeps the loads of RG rows in flight.  BB bounds the block size.  x R = w is solved per thread by
// forward substitution over its instance's columns, from the rows' w values
// exchanged through shared memory.  Grid-stride over pairs of row groups.
// The copy of a new block into the current-block slot is written only when
// the matvec reads it (FP64 matvec); an FP32-matvec batch reads Xf.
template <int RG, int BB>
__global__ void __launch_bounds__(256, 3) k_lz_update_rows(rsed_lanczos_t st, LzDims d, int pass, int crows) {
  extern __shared__ __align__(16) unsigned char smem_u[];
  const int bmax = st.bmax;
  double2* cs = reinterpret_cast<double2*>(smem_u);                    // [(s*bmax + p)][ld]: C[s p][q] of column c0+q
  double2* Rs = cs + (size_t)crows * d.ld;                               // [k*bmax + p][inst]
  double2* wsh = Rs + (size_t)d.n_inst * bmax * bmax;                    // [RG][256] row-group w values
  int* meta = reinterpret_cast<int*>(wsh + RG * 256);                   // [ld]: inst of each column
  for (int c = threadIdx.x; c < d.ld; c += blockDim.x) meta[c] = -1;
  __syncthreads();
  for (int inst = threadIdx.x; inst < d.n_inst; inst += blockDim.x) {
    const int b = st.inst_b[inst], c0 = st.inst_col0[inst];
    for (int q = 0; q < b; ++q) meta[c0 + q] = inst;
  }
  // any_work is the same in every thread (all read the same state words,
  // which no kernel writes meanwhile), so a block with nothing to do (a
  // pass-2 launch after every instance took the single pass) leaves at once
  bool any_work = false;
  for (int inst = 0; inst < d.n_inst; ++inst) {
    const int* stt = st.state + inst * kStateInts;
    const int b = st.inst_b[inst], c0i = st.inst_col0[inst];
    const bool one = stt[S_ONEPASS] != 0;
    const int nb = (pass == 2 || one) ? stt[S_NEWSLOT] : stt[S_NB];
    const double2* coef = reinterpret_cast<const double2*>(st.coef) +
                          (int64_t)inst * 2 * d.pslots * kBMax * kBMax + (pass - 1) * d.pslots * kBMax * kBMax;
    if (!stt[S_ACTIVE] || nb * b > kJacobiMax || (pass == 2 && one)) continue;
    any_work = true;
    for (int e = threadIdx.x; e < nb * b * b; e += blockDim.x) {
      const int r = e / b, q = e % b;  // r = s * b + p
      cs[(size_t)((r / b) * bmax + r % b) * d.ld + c0i + q] = coef[(r / b) * kBMax * kBMax + (r % b) * kBMax + q];
    }
    for (int e = threadIdx.x; e < b * b; e += blockDim.x)
      Rs[((e / b) * bmax + e % b) * d.n_inst + inst] = coef[(d.pslots - 1) * kBMax * kBMax + (e / b) * kBMax + e % b];
  }
  __syncthreads();
  if (!any_work) return;
  const int rows_pg = blockDim.x / d.ld;  // rows per group
  const int rloc = threadIdx.x / d.ld, col = threadIdx.x % d.ld;
  const bool lane_ok = rloc < rows_pg;
  const int inst = lane_ok ? meta[col] : -1;
  int b = 1, c0 = 0, nb = 0, q = 0;
  bool act = false, one = false;
  if (inst >= 0) {
    const int* stt = st.state + inst * kStateInts;
    b = st.inst_b[inst];
    c0 = st.inst_col0[inst];
    one = stt[S_ONEPASS] != 0;
    nb = (pass == 2 || one) ? stt[S_NEWSLOT] : stt[S_NB];
    q = col - c0;
    act = stt[S_ACTIVE] && nb * b <= kJacobiMax && !(pass == 2 && one);
  }
  const double2* ccol = cs + col;                    // C[s p][q] at ccol[(s*bmax + p)*ld]
  const double2* Ri = Rs + (inst < 0 ? 0 : inst);  // R[k][p] at Ri[(k*bmax + p)*n_inst]
  const int ni = d.n_inst;
  double2* V = reinterpret_cast<double2*>(st.V);
  double2* W = reinterpret_cast<double2*>(st.W);
  const int64_t slot_stride = d.n_orb * d.ld;
  const int64_t n_groups = (d.n_orb + rows_pg - 1) / rows_pg;
  const int64_t gstride = (int64_t)rows_pg * d.ld;  // one row group further
  const bool copy_cur = st.Xf == nullptr;  // the FP64 matvec reads the current-block slot
  for (int64_t grp = RG * (int64_t)blockIdx.x; grp < n_groups; grp += RG * (int64_t)gridDim.x) {
    const int64_t row0 = grp * rows_pg + rloc;
    bool live[RG];
    double2 w[RG];
#pragma unroll
    for (int h = 0; h < RG; ++h) {
      live[h] = act && lane_ok && row0 + h * rows_pg < d.n_orb;
      w[h] = make_double2(0.0, 0.0);
    }
    if (live[0]) {
#pragma unroll
      for (int h = 0; h < RG; ++h)
        if (live[h]) w[h] = W[row0 * d.ld + h * gstride + col];
#pragma unroll 2
      for (int s = 0; s < nb; ++s) {
        const double2* Vs = V + s * slot_stride + row0 * d.ld + c0;
#pragma unroll
        for (int p = 0; p < BB; ++p) {
          if (p < b) {
            const double2 c = ccol[(size_t)(s * bmax + p) * d.ld];
#pragma unroll
            for (int h = 0; h < RG; ++h)
              if (live[h]) w[h] = csub(w[h], cmul(Vs[h * gstride + p], c));
          }
        }
      }
    }
#pragma unroll
    for (int h = 0; h < RG; ++h) wsh[h * 256 + threadIdx.x] = w[h];
    __syncthreads();
#pragma unroll
    for (int h = 0; h < RG; ++h) {
      if (!live[h]) continue;
      const int64_t row = row0 + h * rows_pg;
      // forward substitution over this instance's columns 0..q
      const double2* wr = wsh + h * 256 + rloc * d.ld + c0;
      double2 xs[BB];
      double2 xq = make_double2(0.0, 0.0);
#pragma unroll
      for (int pp = 0; pp < BB; ++pp) {
        if (pp > q) break;
        double2 v = wr[pp];
#pragma unroll
        for (int k = 0; k < pp; ++k) v = csub(v, cmul(xs[k], Ri[(k * bmax + pp) * ni]));
        const double rr = Ri[(pp * bmax + pp) * ni].x;
        xs[pp] = make_double2(v.x / rr, v.y / rr);
        xq = xs[pp];
      }
      if (pass == 1 && !one) {
        W[row * d.ld + col] = xq;
      } else {
        V[(int64_t)nb * slot_stride + row * d.ld + col] = xq;
        if (copy_cur) V[(int64_t)(d.n_slots + 1) * slot_stride + row * d.ld + col] = xq;
        if (st.Xf) reinterpret_cast<float2*>(st.Xf)[row * d.ld + col] = make_float2((float)xq.x, (float)xq.y);
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Row-panel streaming forms of the Gram reduction and of the block update.
//
// A panel is pr consecutive rows of one [n_orb][ld] block buffer (W or a basis
// slot): pr * ld * 16 contiguous bytes, at most kPanelElems entries.  A
// streaming block owns the row chunks blockIdx.x, blockIdx.x + gridDim.x, ...
// and walks, per chunk, a fixed sequence of panels (W first, then the slots
// it needs).  Warp kSW (the producer) issues one cp.async.bulk per panel into
// a ring of ns shared-memory stages; the copy completes the stage's "full"
// mbarrier by its byte count.  The kSW consumer warps wait on "full", use the
// panel from shared memory and arrive on the stage's "empty" mbarrier, which
// the producer waits on before it refills the stage.  Every consumer warp
// waits on every panel in order (also on panels it does not use), so a stage
// cannot be refilled before all of them are past it.  With up to ns panels in
// flight per block and two blocks per SM the HBM streams at full rate, and
// the warps do their arithmetic on shared memory with no loads outstanding.
//
// Every mbarrier wait is bounded (kWaitNs of %globaltimer).  A wait that runs
// out raises the block's abort flag; the other warps then stop waiting (they
// still pass every named barrier, so none is left behind), the producer stops
// issuing and waits, bounded again, for the copies it has issued, nothing is
// written, and every instance the block served ends with RSED_ETIMEOUT.
constexpr int kSW = 8;                        // consumer warps
constexpr int kSThreads = (kSW + 1) * 32;     // + the producer warp
constexpr int kPanelElems = 512;              // entries of one panel at most (8 KB)
constexpr int kStreamGridMax = 320;           // streaming blocks at most (Gram partials per instance)
constexpr int kStreamInstMax = 64;            // instances of a streamed batch at most (ld <= 64)
constexpr int kListMax = 2 * kJacobiMax + 8;  // panels of one chunk at most
constexpr unsigned long long kWaitNs = 2000000000ull;
constexpr int kFlagNoStream = 2;              // st.reserved bit 1: use the per-instance kernels
constexpr int kFlagNoStreamUpdate = 4;        // st.reserved bit 2: streamed reduction, row-group update
constexpr int kFlagNoRowRestart = 8;          // st.reserved bit 3: per-instance restart kernel

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// Waits for the completion of the phase with the given parity.  False when the
// block's abort flag is up or the wait ran out of kWaitNs (which raises it).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort) {
  if (*abort) return false;
  if (mbar_test(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (uint32_t it = 1;; ++it) {
    if (mbar_test(bar, parity)) return true;
    if ((it & 63u) == 0) {
      if (*abort) return false;
      if (global_ns() - t0 > kWaitNs) {
        *abort = 1;
        return false;
      }
    }
  }
}
// global -> shared bulk copy of one panel (16-B aligned, multiple of 16 B),
// completing on bar's transaction count
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}
// barrier of the kSW consumer warps only (the producer warp never joins it)
__device__ __forceinline__ void consumer_sync() { asm volatile("bar.sync 1, %0;" ::"n"(kSW * 32) : "memory"); }

// The ring position after a panel: next stage, parity flipped on wrap-around.
__device__ __forceinline__ void ring_next(int& stg, uint32_t& ph, int ns) {
  if (++stg == ns) {
    stg = 0;
    ph ^= 1u;
  }
}

// After an abort: waits, bounded, for the last copy issued into each stage.
__device__ void stream_drain(uint64_t* full, int ns, int64_t issued) {
  for (int64_t k = issued > ns ? issued - ns : 0; k < issued; ++k) {
    const int stg = (int)(k % ns);
    const uint32_t par = (uint32_t)((k / ns) & 1);
    const uint64_t t0 = global_ns();
    while (!mbar_test(&full[stg], par) && global_ns() - t0 < kWaitNs) {
    }
  }
}

struct StreamLayout {
  size_t bars, ring, wl, coef, rs, total;
};
// dynamic shared memory of a streaming block: ns full + ns empty barriers,
// the ring, one panel-sized work buffer, the coefficients (column-major:
// crows rows of ld columns, so the lanes of a warp read consecutive words)
// and, for the update, the instances' R factors ([k][p][instance])
__host__ __device__ inline StreamLayout stream_layout(int ns, int n_inst, int crows, int ld, bool with_r) {
  StreamLayout l;
  size_t off = 0;
  l.bars = off;
  off += 16 * (size_t)ns;
  off = (off + 127) & ~(size_t)127;
  l.ring = off;
  off += sizeof(double2) * kPanelElems * (size_t)ns;
  l.wl = off;
  off += sizeof(double2) * kPanelElems;
  l.coef = off;
  off += sizeof(double2) * (size_t)crows * ld;
  l.rs = off;
  off += with_r ? sizeof(double2) * (size_t)n_inst * kBMax * kBMax : 0;
  l.total = off;
  return l;
}

// The producer: lane 0 of warp kSW issues the block's panels in order.
// list[t] names panel t of a chunk: -1 = W, s >= 0 = basis slot s.
__device__ void stream_produce(const rsed_lanczos_t& st, const LzDims& d, int ns, int pr, const int* list, int npc,
                               int64_t my_chunks, uint64_t* full, uint64_t* empty, double2* ring,
                               volatile int* abort) {
  const double2* V = reinterpret_cast<const double2*>(st.V);
  const double2* W = reinterpret_cast<const double2*>(st.W);
  const int64_t slot_stride = d.n_orb * d.ld;
  const int64_t total = my_chunks * npc;
  int64_t issued = 0;
  int stg = 0, t = 0;
  uint32_t ph = 0;  // parity of this stage's current use
  int64_t r0 = (int64_t)blockIdx.x * pr;
  for (int64_t k = 0; k < total; ++k) {
    // the stage's previous use (panel k - ns) must be released by every consumer
    if (k >= ns && !mbar_wait(&empty[stg], ph ^ 1u, abort)) break;
    const int64_t rows = min((int64_t)pr, d.n_orb - r0);
    const int sl = list[t];
    const double2* src = (sl < 0 ? W : V + (int64_t)sl * slot_stride) + r0 * d.ld;
    const uint32_t bytes = (uint32_t)(rows * d.ld * (int64_t)sizeof(double2));
    mbar_expect_tx(&full[stg], bytes);
    bulk_load(ring + (size_t)stg * kPanelElems, src, bytes, &full[stg]);
    issued = k + 1;
    ring_next(stg, ph, ns);
    if (++t == npc) {
      t = 0;
      r0 += (int64_t)gridDim.x * pr;
    }
  }
  if (*abort) stream_drain(full, ns, issued);
}

// Gram partials of all instances over the block's row chunks:
//   partial[blk][inst][s][p][q] = sum_rows conj(Y_s[row][c0+p]) W_loc[row][c0+q]
// with Y_s = V[s] for s < nb and Y_nb = W_loc (the finalisation, k_lz_finalize,
// sums the gridDim.x partials).  Per chunk: W and the slots the local
// transform needs are streamed first and W_loc is formed element-wise into
// shared memory (thread = entry of the panel); then every basis slot s < max
// nb is streamed, and warp s % kSW adds it into its registers (lane = column
// c0 + p, all q of the instance), reading W_loc from shared memory.  BB is
// the largest block of the batch rounded up to a power of two, CPL the
// columns per lane (ld <= 32 * CPL).
template <int BB, int CPL>
__global__ void __launch_bounds__(kSThreads, 2)
    k_lz_gram_stream(rsed_lanczos_t st, LzDims d, int pass, int ns, int pr, int crows) {
  constexpr int SW = kJacobiMax / BB / kSW + 1;  // slots one warp owns at most
  extern __shared__ __align__(128) unsigned char smem_s[];
  const StreamLayout L = stream_layout(ns, d.n_inst, crows, d.ld, false);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_s + L.bars);
  uint64_t* empty = full + ns;
  double2* ring = reinterpret_cast<double2*>(smem_s + L.ring);
  double2* wl = reinterpret_cast<double2*>(smem_s + L.wl);
  double2* lc = reinterpret_cast<double2*>(smem_s + L.coef);
  __shared__ int s_b[kStreamInstMax], s_c0[kStreamInstMax], s_nb[kStreamInstMax], s_jloc[kStreamInstMax];
  __shared__ unsigned long long s_lnz[kStreamInstMax];
  __shared__ double s_sig[32 * CPL];  // sigma of each column
  __shared__ int s_col_inst[32 * CPL];
  __shared__ int s_list[kListMax];
  __shared__ int s_npc, s_nloc, s_nbmax;
  __shared__ int s_abort_store;
  volatile int* s_abort = &s_abort_store;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ld = d.ld;
  if (tid == 0) s_abort_store = 0;
  for (int c = tid; c < 32 * CPL; c += kSThreads) s_col_inst[c] = -1;
  __syncthreads();
  for (int i = tid; i < d.n_inst; i += kSThreads) {
    const int* stt = st.state + i * kStateInts;
    const int b = st.inst_b[i], c0 = st.inst_col0[i], nb = stt[S_NB];
    const bool valid = nb <= d.n_slots && b >= 1 && b <= kBMax && nb * b <= kJacobiMax + kBMax;
    const bool act = stt[S_ACTIVE] && !(pass == 2 && stt[S_ONEPASS]) && valid;
    s_b[i] = b;
    s_c0[i] = c0;
    s_nb[i] = act ? nb : -1;
    s_jloc[i] = (act && pass == 1 && nb >= 2 && (st.reserved & kFlagSinglePass)) ? nb - 1 : 0;
    if (act)
      for (int q = 0; q < b; ++q) s_col_inst[c0 + q] = i;
  }
  __syncthreads();
  // the known part of the recurrence per instance (pass 1, single pass on):
  // lc[(l*bmax + p)*ld + c0 + q] = conj(P[j*b + q][l*b + p]) for l < j = nb - 1,
  // sigma of column c0 + q = Re P[(j-1)*b + q][(j-1)*b + q]
  const int bmax = st.bmax;
  for (int i = 0; i < d.n_inst; ++i) {
    const int jl = s_jloc[i];
    if (jl == 0) continue;
    const int b = s_b[i], c0 = s_c0[i];
    const double2* Pi = reinterpret_cast<const double2*>(st.P) + (int64_t)i * d.pm * d.pm;
    for (int e = tid; e < jl * b * b; e += kSThreads) {
      const int r = e / b, q = e % b;  // r = l*b + p
      lc[(size_t)((r / b) * bmax + r % b) * ld + c0 + q] = cconj(Pi[(int64_t)(jl * b + q) * d.pm + r]);
    }
    if (tid < b) s_sig[c0 + tid] = Pi[(int64_t)((jl - 1) * b + tid) * d.pm + (jl - 1) * b + tid].x;
  }
  __syncthreads();
  for (int i = tid; i < d.n_inst; i += kSThreads) {
    unsigned long long m = 0;
    const int jl = s_jloc[i], b = s_b[i], c0 = s_c0[i];
    for (int l = 0; l < jl; ++l) {
      bool nz = false;
      for (int e = 0; e < b * b; ++e) {
        const double2 v = lc[(size_t)(l * bmax + e / b) * ld + c0 + e % b];
        nz |= (v.x != 0.0) || (v.y != 0.0);
      }
      if (nz) m |= 1ull << l;
    }
    s_lnz[i] = m;
  }
  __syncthreads();
  if (tid == 0) {
    int nbmax = -1;
    unsigned long long need = 0;
    for (int i = 0; i < d.n_inst; ++i) {
      nbmax = max(nbmax, s_nb[i]);
      if (s_jloc[i]) need |= s_lnz[i] | (1ull << s_jloc[i]);
    }
    int n = 0;
    s_list[n++] = -1;
    for (int l = 0; l < 64; ++l)
      if ((need >> l) & 1ull) s_list[n++] = l;
    s_nloc = n - 1;
    for (int s = 0; s < nbmax; ++s) s_list[n++] = s;
    s_npc = n;
    s_nbmax = nbmax;
    for (int k = 0; k < ns; ++k) {
      mbar_init(&full[k], 1);
      mbar_init(&empty[k], kSW);
    }
    mbar_init_fence();
  }
  __syncthreads();
  const int nbmax = s_nbmax;
  if (nbmax < 0) return;  // no instance has work in this pass
  const int npc = s_npc, nloc = s_nloc;
  const int64_t n_rchunks = (d.n_orb + pr - 1) / pr;
  const int64_t my_chunks = blockIdx.x < n_rchunks ? (n_rchunks - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  if (warp == kSW) {
    if (lane == 0) stream_produce(st, d, ns, pr, s_list, npc, my_chunks, full, empty, ring, s_abort);
  } else {
    double2 acc[SW][CPL][BB];
#pragma unroll
    for (int j = 0; j < SW; ++j)
#pragma unroll
      for (int c = 0; c < CPL; ++c)
#pragma unroll
        for (int q = 0; q < BB; ++q) acc[j][c][q] = make_double2(0.0, 0.0);
    // this lane's columns (Gram) and this thread's two entries (W_loc)
    int cinst[CPL], cnb[CPL], cb[CPL], cc0[CPL];
#pragma unroll
    for (int c = 0; c < CPL; ++c) {
      const int col = lane + 32 * c;
      const int i = col < ld ? s_col_inst[col] : -1;
      cinst[c] = i;
      cnb[c] = i >= 0 ? s_nb[i] : -1;
      cb[c] = i >= 0 ? s_b[i] : 0;
      cc0[c] = i >= 0 ? s_c0[i] : 0;
    }
    int einst[2], erow[2], ecol[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int e = tid + u * kSW * 32;
      erow[u] = e / ld;
      ecol[u] = e % ld;
      einst[u] = (erow[u] < pr) ? s_col_inst[ecol[u]] : -1;
    }
    int stg = 0;      // ring stage of the next panel
    uint32_t ph = 0;  // parity of that stage's current use
    for (int64_t ci = 0; ci < my_chunks; ++ci) {
      const int64_t r0 = (blockIdx.x + ci * gridDim.x) * (int64_t)pr;
      const int rows = (int)min((int64_t)pr, d.n_orb - r0);
      double2 w[2];
      {
        mbar_wait(&full[stg], ph, s_abort);
        const double2* pnl = ring + (size_t)stg * kPanelElems;
#pragma unroll
        for (int u = 0; u < 2; ++u) w[u] = erow[u] < rows ? pnl[erow[u] * ld + ecol[u]] : make_double2(0.0, 0.0);
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[stg]);
        ring_next(stg, ph, ns);
      }
      for (int t = 1; t <= nloc; ++t) {
        const int sl = s_list[t];
        mbar_wait(&full[stg], ph, s_abort);
        const double2* pnl = ring + (size_t)stg * kPanelElems;
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const int i = einst[u];
          if (i < 0 || erow[u] >= rows) continue;
          const int jl = s_jloc[i];
          if (jl == 0) continue;
          const int b = s_b[i], c0 = s_c0[i];
          const double2* prow = pnl + erow[u] * ld + c0;
          if (sl == jl) {
            const double2 x = pnl[erow[u] * ld + ecol[u]];
            w[u].x -= s_sig[ecol[u]] * x.x;
            w[u].y -= s_sig[ecol[u]] * x.y;
          } else if (sl < jl && ((s_lnz[i] >> sl) & 1ull)) {
            const double2* Lc = lc + (size_t)sl * bmax * ld + ecol[u];
            for (int p = 0; p < b; ++p) w[u] = csub(w[u], cmul(prow[p], Lc[p * ld]));
          }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[stg]);
        ring_next(stg, ph, ns);
      }
      consumer_sync();  // every warp is done with the previous chunk's W_loc
#pragma unroll
      for (int u = 0; u < 2; ++u)
        if (erow[u] < pr) wl[erow[u] * ld + ecol[u]] = w[u];
      consumer_sync();
      // Gram of W_loc itself: slot nb of the lane's instance
#pragma unroll
      for (int c = 0; c < CPL; ++c) {
        if (cinst[c] < 0) continue;
        const int col = lane + 32 * c;
#pragma unroll
        for (int jj = 0; jj < SW; ++jj) {
          if (cnb[c] != jj * kSW + warp) continue;
          for (int r = 0; r < rows; ++r) {
            const double2 y = wl[r * ld + col];
            const double2* wr = wl + r * ld + cc0[c];
#pragma unroll
            for (int q = 0; q < BB; ++q)
              if (q < cb[c]) acc[jj][c][q] = cadd(acc[jj][c][q], cdotc(y, wr[q]));
          }
        }
      }
      // basis slots 0 .. nbmax-1, slot s added by warp s % kSW
#pragma unroll
      for (int jj = 0; jj < SW; ++jj) {
        for (int ww = 0; ww < kSW; ++ww) {
          const int s = jj * kSW + ww;
          if (s >= nbmax) break;
          mbar_wait(&full[stg], ph, s_abort);
          if (ww == warp) {
            const double2* pnl = ring + (size_t)stg * kPanelElems;
#pragma unroll
            for (int c = 0; c < CPL; ++c) {
              if (s >= cnb[c]) continue;
              const int col = lane + 32 * c;
#pragma unroll 4
              for (int r = 0; r < rows; ++r) {
                const double2 y = pnl[r * ld + col];
                const double2* wr = wl + r * ld + cc0[c];
#pragma unroll
                for (int q = 0; q < BB; ++q)
                  if (q < cb[c]) acc[jj][c][q] = cadd(acc[jj][c][q], cdotc(y, wr[q]));
              }
            }
          }
          __syncwarp();
          if (lane == 0) mbar_arrive(&empty[stg]);
          ring_next(stg, ph, ns);
        }
      }
    }
    if (!*s_abort) {
      double2* part = reinterpret_cast<double2*>(st.partial);
#pragma unroll
      for (int c = 0; c < CPL; ++c) {
        const int i = cinst[c];
        if (i < 0) continue;
        const int p = lane + 32 * c - cc0[c];
#pragma unroll
        for (int jj = 0; jj < SW; ++jj) {
          const int s = jj * kSW + warp;
          if (s > cnb[c]) continue;
          double2* out = part + (((int64_t)blockIdx.x * d.n_inst + i) * d.pslots + s) * kBMax * kBMax + p * kBMax;
#pragma unroll
          for (int q = 0; q < BB; ++q)
            if (q < cb[c]) out[q] = acc[jj][c][q];
        }
      }
    }
  }
  __syncthreads();
  if (*s_abort && tid == 0) {
    for (int i = 0; i < d.n_inst; ++i) {
      if (s_nb[i] < 0) continue;
      int* stt = st.state + i * kStateInts;
      stt[S_STATUS] = RSED_ETIMEOUT;
      stt[S_ACTIVE] = 0;
    }
  }
}

// Finalisation of the streamed Gram partials, one block per instance (the
// same arithmetic as the last block of k_lz_reduce).
__global__ void __launch_bounds__(kRT) k_lz_finalize(rsed_lanczos_t st, LzDims d, int pass) {
  const int inst = blockIdx.x;
  int* stt = st.state + inst * kStateInts;
  if (pass == 1 && threadIdx.x == 0) stt[S_RESTART_NB] = 0;
  if (!stt[S_ACTIVE]) return;
  if (pass == 2 && stt[S_ONEPASS]) return;
  const int b = st.inst_b[inst];
  const int nb = stt[S_NB];
  __shared__ int s_ok, s_one;
  __shared__ double2 sc[(kJacobiMax / 1 + kBMax + kBMax) * kBMax];
  __shared__ double2 sR[kBMax * kBMax];
  __shared__ double2 sG[kBMax * kBMax];
  __shared__ double2 fin[kRT * kBMax];
  if (nb > d.n_slots || b < 1 || b > kBMax || nb * b > kJacobiMax + kBMax) {
    if (threadIdx.x == 0) {
      stt[S_STATUS] = RSED_EINVAL;
      stt[S_ACTIVE] = 0;
    }
    return;
  }
  const bool loc = pass == 1 && nb >= 2 && (st.reserved & kFlagSinglePass);
  lz_finalize(st, d, inst, pass, b, nb, stt, sc, sR, sG, &s_ok, fin, loc, &s_one);
}

// W <- (W_loc - V C) R^-1 for all instances, streamed: per chunk W and the
// basis slots s < max nb; thread = entry (row, column c0 + q) of the panel,
// subtracting sum_p V_s[row][c0+p] C[s p][q] from shared memory; the rows are
// then solved with R by forward substitution over the instance's columns
// (exchanged through shared memory) and stored as in k_lz_update_rows.
__global__ void __launch_bounds__(kSThreads, 2)
    k_lz_update_stream(rsed_lanczos_t st, LzDims d, int pass, int ns, int pr, int crows) {
  extern __shared__ __align__(128) unsigned char smem_s[];
  const StreamLayout L = stream_layout(ns, d.n_inst, crows, d.ld, true);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_s + L.bars);
  uint64_t* empty = full + ns;
  double2* ring = reinterpret_cast<double2*>(smem_s + L.ring);
  double2* wsh = reinterpret_cast<double2*>(smem_s + L.wl);
  double2* cs = reinterpret_cast<double2*>(smem_s + L.coef);
  double2* Rs = reinterpret_cast<double2*>(smem_s + L.rs);
  __shared__ int s_b[kStreamInstMax], s_c0[kStreamInstMax], s_nb[kStreamInstMax], s_one[kStreamInstMax];
  __shared__ int s_col_inst[64];
  __shared__ int s_list[kJacobiMax + 2];
  __shared__ int s_nbmax;
  __shared__ int s_abort_store;
  volatile int* s_abort = &s_abort_store;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ld = d.ld;
  if (tid == 0) s_abort_store = 0;
  for (int c = tid; c < 64; c += kSThreads) s_col_inst[c] = -1;
  __syncthreads();
  for (int i = tid; i < d.n_inst; i += kSThreads) {
    const int* stt = st.state + i * kStateInts;
    const int b = st.inst_b[i], c0 = st.inst_col0[i];
    const bool one = stt[S_ONEPASS] != 0;
    const int nb = (pass == 2 || one) ? stt[S_NEWSLOT] : stt[S_NB];
    const bool act = stt[S_ACTIVE] && b >= 1 && b <= kBMax && nb * b <= kJacobiMax && !(pass == 2 && one);
    s_b[i] = b;
    s_c0[i] = c0;
    s_one[i] = one;
    s_nb[i] = act ? nb : -1;
    if (act)
      for (int q = 0; q < b; ++q) s_col_inst[c0 + q] = i;
  }
  __syncthreads();
  // cs[(s*bmax + p)*ld + c0 + q] = C[s p][q], Rs[(k*kBMax + p)*n_inst + i] = R_i[k][p]
  const int bmax = st.bmax;
  for (int i = 0; i < d.n_inst; ++i) {
    const int nb = s_nb[i], b = s_b[i], c0 = s_c0[i];
    if (nb < 0) continue;
    const double2* coef = reinterpret_cast<const double2*>(st.coef) +
                          (int64_t)i * 2 * d.pslots * kBMax * kBMax + (pass - 1) * d.pslots * kBMax * kBMax;
    for (int e = tid; e < nb * b * b; e += kSThreads) {
      const int r = e / b, q = e % b;  // r = s * b + p
      cs[(size_t)((r / b) * bmax + r % b) * ld + c0 + q] = coef[(r / b) * kBMax * kBMax + (r % b) * kBMax + q];
    }
    for (int e = tid; e < kBMax * kBMax; e += kSThreads)
      Rs[e * d.n_inst + i] = coef[(d.pslots - 1) * kBMax * kBMax + e];
  }
  if (tid == 0) {
    int nbmax = -1;
    for (int i = 0; i < d.n_inst; ++i) nbmax = max(nbmax, s_nb[i]);
    s_list[0] = -1;
    for (int s = 0; s < nbmax; ++s) s_list[1 + s] = s;
    s_nbmax = nbmax;
    for (int k = 0; k < ns; ++k) {
      mbar_init(&full[k], 1);
      mbar_init(&empty[k], kSW);
    }
    mbar_init_fence();
  }
  __syncthreads();
  const int nbmax = s_nbmax;
  if (nbmax < 0) return;
  const int npc = 1 + nbmax;
  const int64_t n_rchunks = (d.n_orb + pr - 1) / pr;
  const int64_t my_chunks = blockIdx.x < n_rchunks ? (n_rchunks - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  if (warp == kSW) {
    if (lane == 0) stream_produce(st, d, ns, pr, s_list, npc, my_chunks, full, empty, ring, s_abort);
  } else {
    double2* V = reinterpret_cast<double2*>(st.V);
    double2* W = reinterpret_cast<double2*>(st.W);
    const int64_t slot_stride = d.n_orb * d.ld;
    const bool copy_cur = st.Xf == nullptr;  // the FP64 matvec reads the current-block slot
    int einst[2], erow[2], ecol[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int e = tid + u * kSW * 32;
      erow[u] = e / ld;
      ecol[u] = e % ld;
      einst[u] = (erow[u] < pr) ? s_col_inst[ecol[u]] : -1;
    }
    int stg = 0;      // ring stage of the next panel
    uint32_t ph = 0;  // parity of that stage's current use
    for (int64_t ci = 0; ci < my_chunks; ++ci) {
      const int64_t r0 = (blockIdx.x + ci * gridDim.x) * (int64_t)pr;
      const int rows = (int)min((int64_t)pr, d.n_orb - r0);
      double2 w[2];
      {
        mbar_wait(&full[stg], ph, s_abort);
        const double2* pnl = ring + (size_t)stg * kPanelElems;
#pragma unroll
        for (int u = 0; u < 2; ++u) w[u] = erow[u] < rows ? pnl[erow[u] * ld + ecol[u]] : make_double2(0.0, 0.0);
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[stg]);
        ring_next(stg, ph, ns);
      }
#pragma unroll 2
      for (int s = 0; s < nbmax; ++s) {
        mbar_wait(&full[stg], ph, s_abort);
        const double2* pnl = ring + (size_t)stg * kPanelElems;
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const int i = einst[u];
          if (i < 0 || erow[u] >= rows || s >= s_nb[i]) continue;
          const int b = s_b[i], c0 = s_c0[i];
          const double2* prow = pnl + erow[u] * ld + c0;
          const double2* ccol = cs + (size_t)s * bmax * ld + ecol[u];
          for (int p = 0; p < b; ++p) w[u] = csub(w[u], cmul(prow[p], ccol[p * ld]));
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[stg]);
        ring_next(stg, ph, ns);
      }
      consumer_sync();  // every warp is done with the previous chunk's rows
#pragma unroll
      for (int u = 0; u < 2; ++u)
        if (erow[u] < pr) wsh[erow[u] * ld + ecol[u]] = w[u];
      consumer_sync();
      if (*s_abort) continue;
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int i = einst[u];
        if (i < 0 || erow[u] >= rows) continue;
        const int b = s_b[i], c0 = s_c0[i], q = ecol[u] - c0, nb = s_nb[i];
        const double2* wr = wsh + erow[u] * ld + c0;
        const double2* Ri = Rs + i;  // R_i[k][p] at Ri[(k*kBMax + p)*n_inst]
        const int ni = d.n_inst;
        double2 xs[kBMax];
        double2 xq = make_double2(0.0, 0.0);
#pragma unroll
        for (int pp = 0; pp < kBMax; ++pp) {
          if (pp > q) break;
          double2 v = wr[pp];
          for (int kq = 0; kq < pp; ++kq) v = csub(v, cmul(xs[kq], Ri[(kq * kBMax + pp) * ni]));
          const double rr = Ri[(pp * kBMax + pp) * ni].x;
          xs[pp] = make_double2(v.x / rr, v.y / rr);
          xq = xs[pp];
        }
        (void)b;
        const int64_t at = (r0 + erow[u]) * ld + ecol[u];
        if (pass == 1 && !s_one[i]) {
          W[at] = xq;
        } else {
          V[(int64_t)nb * slot_stride + at] = xq;
          if (copy_cur) V[(int64_t)(d.n_slots + 1) * slot_stride + at] = xq;
          if (st.Xf) reinterpret_cast<float2*>(st.Xf)[at] = make_float2((float)xq.x, (float)xq.y);
        }
      }
    }
  }
  __syncthreads();
  if (*s_abort && tid == 0) {
    for (int i = 0; i < d.n_inst; ++i) {
      if (s_nb[i] < 0) continue;
      int* stt = st.state + i * kStateInts;
      stt[S_STATUS] = RSED_ETIMEOUT;
      stt[S_ACTIVE] = 0;
    }
  }
}

// ---------------------------------------------------------------------------
// Lowest Kp eigenpairs of a Hermitian M x M matrix held in shared memory
// (full row-major storage, destroyed), one thread block:
//   1. Householder reduction to a real symmetric tridiagonal T = Q^H A Q
//      (lower variant of LAPACK zhetd2: reflectors H_k = I - tau_k v v^H
//      chosen so the sub-diagonal comes out real), ~5 block barriers per column;
//   2. eigenvalues of T by Sturm-sequence bisection, one thread per eigenvalue;
//   3. eigenvectors of T by inverse iteration (tridiagonal LU with partial
//      pivoting, three solves), one thread per eigenvector, then modified
//      Gram-Schmidt in ascending order (orthonormal bases of degenerate
//      clusters);
//   4. back-transformation s = H_0 H_1 ... H_{M-2} z, one warp per vector.
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Number of eigenvalues of the symmetric tridiagonal (d, e) below x, by
// Sturm's theorem on the leading principal minors p_{-1} = 1,
// p_i = (d_i - x) p_{i-1} - e_{i-1}^2 p_{i-2} (the recurrence of Wilkinson's
// bisection, 1962): a sign change between consecutive minors is a negative
// pivot q_i = p_i / p_{i-1}, and the recurrence needs no division.
// de[i] = (d_i, e_i^2) and x come scaled by one power of two so that
// |d_i| + |e_i| <= 1 (exact: every sign and rounding is the unscaled one);
// the two live minors are rescaled by a power of two whenever the newer one
// leaves [2^-400, 2^400].  A minor that vanishes against its predecessor,
// |p_i| < piv |p_{i-1}|, becomes -piv p_{i-1} (the pivmin rule of the ratio
// form).  piv >= 2^-500 keeps piv |p_{i-1}| a normal number.
__device__ int sturm_count(const double2* de, int M, double x, double piv) {
  double pm = de[0].x - x;  // p_0
  if (fabs(pm) < piv) pm = -piv;
  int c = pm < 0.0;
  double pmm = 1.0;  // p_{-1}
  for (int i = 1; i < M; ++i) {
    const double2 v = de[i];
    const double t = de[i - 1].y * pmm;
    double p = fma(v.x - x, pm, -t);
    if (fabs(p) < piv * fabs(pm)) p = -piv * pm;
    c += (p < 0.0) != (pm < 0.0);
    pmm = pm;
    pm = p;
    if (!(fabs(pm) <= 0x1p400 && fabs(pm) >= 0x1p-400)) {
      int ex;
      frexp(pm, &ex);
      pm = ldexp(pm, -ex);
      pmm = ldexp(pmm, -ex);
    }
  }
  return c;
}

// Householder reflector of column c (rows c+1..M-1) by one warp: v (v[c+1] =
// 1) into A's column c and into vb, tau[c], the off-diagonal ee[c].
__device__ __forceinline__ void herm_reflector(double2* A, int lda, int M, int c, double2* vb, double2* tau,
                                               double* ee, int lane) {
  double sq = 0.0;
  for (int i = c + 2 + lane; i < M; i += 32) {
    const double2 v = A[i * lda + c];
    sq += v.x * v.x + v.y * v.y;
  }
  sq = warp_sum(sq);
  const double2 al = A[(c + 1) * lda + c];
  double2 t = make_double2(0.0, 0.0), scl = make_double2(0.0, 0.0);
  double beta = al.x;
  if (sq != 0.0 || al.y != 0.0) {
    beta = -copysign(sqrt(al.x * al.x + al.y * al.y + sq), al.x);
    const double ib = 1.0 / beta;
    t = make_double2((beta - al.x) * ib, -al.y * ib);
    const double2 den = make_double2(al.x - beta, al.y);
    const double idn = 1.0 / (den.x * den.x + den.y * den.y);
    scl = make_double2(den.x * idn, -den.y * idn);
  }
  for (int i = c + 2 + lane; i < M; i += 32) {
    const double2 v = cmul(A[i * lda + c], scl);
    A[i * lda + c] = v;
    vb[i] = v;
  }
  if (lane == 0) {
    vb[c + 1] = make_double2(1.0, 0.0);
    A[(c + 1) * lda + c] = make_double2(1.0, 0.0);
    tau[c] = t;
    ee[c] = beta;
  }
  __syncwarp();
}

// iwork: optional shared-memory work area of kHermWork bytes for the inverse
// iteration (NULL: thread-local arrays).
__device__ void herm_lowest(double2* A, int M, int Kp, double* theta, double2* S, double* Z, double2* tau,
                            double* dd, double* ee, double* red, double2* vv, double2* pw, double* iwork) {
  // A is M x M with row stride lda = M + 1 (odd, so column walks hit distinct banks)
  const int lda = M + 1;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nwarp = nt >> 5;
  // ---- 1. tridiagonalisation: two barriers per column ----
  // Warp 0 updates column k+1 itself during step k's rank-2 update and forms
  // the next reflector at once (look-ahead), while the other warps update the
  // rest of the trailing matrix; the reflector vectors alternate between two
  // buffers (vv and the still unused S), so the next one never overwrites the
  // one being applied.  p^H v is formed redundantly by every warp.
  double2* vbuf[2] = {vv, S};
  if (M >= 2 && warp == 0) herm_reflector(A, lda, M, 0, vbuf[0], tau, ee, lane);
  __syncthreads();
  for (int k = 0; k < M - 1; ++k) {
    const double2* v = vbuf[k & 1];
    const double2 t = tau[k];
    const bool next = k + 1 < M - 1;
    if (t.x == 0.0 && t.y == 0.0) {  // H_k = I: nothing to update
      if (next && warp == 0) herm_reflector(A, lda, M, k + 1, vbuf[(k + 1) & 1], tau, ee, lane);
      __syncthreads();
      continue;
    }
    // p = tau * A22 v, four lanes per row
    {
      const int i = k + 1 + (tid >> 2), sub = tid & 3;
      double sx = 0.0, sy = 0.0;
      if (i < M) {
        const double2* Ar = A + i * lda;
        for (int j = k + 1 + sub; j < M; j += 4) {
          const double2 a = Ar[j], vj = v[j];
          sx += a.x * vj.x - a.y * vj.y;
          sy += a.x * vj.y + a.y * vj.x;
        }
      }
      sx += __shfl_xor_sync(0xffffffffu, sx, 1);
      sy += __shfl_xor_sync(0xffffffffu, sy, 1);
      sx += __shfl_xor_sync(0xffffffffu, sx, 2);
      sy += __shfl_xor_sync(0xffffffffu, sy, 2);
      if (i < M && sub == 0) pw[i] = cmul(t, make_double2(sx, sy));
    }
    __syncthreads();
    // p^H v in every warp; alpha = -1/2 tau (p^H v); w = p + alpha v
    double2 alpha;
    {
      double sx = 0.0, sy = 0.0;
      for (int i = k + 1 + lane; i < M; i += 32) {
        const double2 c = cdotc(pw[i], v[i]);
        sx += c.x;
        sy += c.y;
      }
      const double2 ta = cmul(t, make_double2(warp_sum(sx), warp_sum(sy)));
      alpha = make_double2(-0.5 * ta.x, -0.5 * ta.y);
    }
    // A22 -= v w^H + w v^H: column k+1 by warp 0 (then the next reflector),
    // columns k+2.. of every row by the other warps (all warps if there is one)
    const int c1 = k + 1;
    const double2 v1 = v[c1];
    const double2 w1 = cadd(pw[c1], cmul(alpha, v1));
    if (warp == 0) {
      for (int i = c1 + lane; i < M; i += 32) {
        const double2 vi = v[i];
        const double2 wi = cadd(pw[i], cmul(alpha, vi));
        const double2 u = cadd(make_double2(vi.x * w1.x + vi.y * w1.y, vi.y * w1.x - vi.x * w1.y),
                               make_double2(wi.x * v1.x + wi.y * v1.y, wi.y * v1.x - wi.x * v1.y));
        A[i * lda + c1] = csub(A[i * lda + c1], u);
      }
      __syncwarp();
      if (next) herm_reflector(A, lda, M, c1, vbuf[c1 & 1], tau, ee, lane);
    }
    const int w0 = nwarp > 1 ? 1 : 0, nw = nwarp > 1 ? nwarp - 1 : 1;
    if (warp >= w0) {
      for (int i = c1 + (warp - w0); i < M; i += nw) {
        const double2 vi = v[i];
        const double2 wi = cadd(pw[i], cmul(alpha, vi));
        for (int j = c1 + 1 + lane; j < M; j += 32) {
          const double2 vj = v[j];
          const double2 wj = cadd(pw[j], cmul(alpha, vj));
          const double2 u = cadd(make_double2(vi.x * wj.x + vi.y * wj.y, vi.y * wj.x - vi.x * wj.y),
                                 make_double2(wi.x * vj.x + wi.y * vj.y, wi.y * vj.x - wi.x * vj.y));
          A[i * lda + j] = csub(A[i * lda + j], u);
        }
      }
    }
    __syncthreads();
  }
  for (int k = tid; k < M; k += nt) dd[k] = A[k * lda + k].x;
  if (tid == 0 && M >= 1) ee[M - 1] = 0.0;
  __syncthreads();
  // ---- 2. eigenvalues: 16-way multisection, 16 threads per eigenvalue ----
  double lo = 1e300, hi = -1e300, emax2 = 0.0;
  for (int i = 0; i < M; ++i) {
    const double r = (i > 0 ? fabs(ee[i - 1]) : 0.0) + (i < M - 1 ? fabs(ee[i]) : 0.0);
    lo = fmin(lo, dd[i] - r);
    hi = fmax(hi, dd[i] + r);
    if (i < M - 1) emax2 = fmax(emax2, ee[i] * ee[i]);
  }
  const double tnorm = fmax(fabs(lo), fabs(hi));
  const double pivmin = 1e-300 * fmax(1.0, emax2);
  // (d_i, e_i^2) scaled by 2^-ks (|d_i| + |e_i| <= tnorm < 2^ks) into pw, free
  // since the tridiagonalisation, for the division-free Sturm counts
  int ks;
  frexp(tnorm, &ks);
  for (int i = tid; i < M; i += nt) {
    const double es = ldexp(ee[i], -ks);
    pw[i] = make_double2(ldexp(dd[i], -ks), es * es);
  }
  const double piv = fmax(ldexp(pivmin, -ks), 0x1p-500);
  __syncthreads();
  {
    const int j = tid >> 4, sub = tid & 15;  // eigenvalue j, sample point sub
    double a = lo - 1e-12 * tnorm - 1e-300, bnd = hi + 1e-12 * tnorm + 1e-300;
    // 16 rounds shrink the Gershgorin interval by 16^16 ~ 1.8e19: below one ulp.
    // A warp stops early once both its brackets are down to rounding level
    // (decided by __all_sync, so every lane of the warp stays in the ballot).
    for (int round = 0; round < 16; ++round) {
      if (__all_sync(0xffffffffu, bnd - a <= 4e-16 * fmax(fabs(a), fabs(bnd)) + pivmin)) break;
      const double w = (bnd - a) * (1.0 / 16.0);
      const double x = a + w * (sub + 1);
      const int c = (j < Kp && sub < 15) ? sturm_count(pw, M, ldexp(x, -ks), piv) : 1 << 30;
      // first sample whose count exceeds j bounds the eigenvalue from above
      const unsigned ballot = __ballot_sync(0xffffffffu, c > j);
      const unsigned mine = (ballot >> ((lane >> 4) << 4)) & 0xFFFFu;
      const int first = __ffs(mine) - 1;  // 0..15 (15 = the upper end)
      const double na = a + w * first;
      bnd = a + w * (first + 1);
      a = na;
    }
    if (j < Kp && sub == 0) theta[j] = 0.5 * (a + bnd);
  }
  __syncthreads();
  // ---- 3. inverse iteration ----
  if (tid < Kp) {
    const int j = tid;
    double lam = theta[j];
    const double sep = 1e-14 * fmax(tnorm, 1e-300);
    for (int i = 0; i < j; ++i)  // separate shifts of (nearly) equal eigenvalues
      if (fabs(lam - theta[i]) < sep) lam = theta[i] + sep * (j - i + 1);
    // the vector's work arrays: in the shared work area, element i of vector
    // j at i * Kp + j (the Kp threads touch consecutive words), else local
    double ldl[kJacobiMax], ldg[kJacobiMax], ldu[kJacobiMax], ldu2[kJacobiMax], lz[kJacobiMax];
    unsigned char lpiv[kJacobiMax];
    const int sw = iwork ? Kp : 1;
    const int mk = kJacobiMax * kKeepMax;
    double* dlp = iwork ? iwork + j : ldl;
    double* dgp = iwork ? iwork + mk + j : ldg;
    double* dup = iwork ? iwork + 2 * mk + j : ldu;
    double* du2p = iwork ? iwork + 3 * mk + j : ldu2;
    double* zp = iwork ? iwork + 4 * mk + j : lz;
    unsigned char* pivp = iwork ? reinterpret_cast<unsigned char*>(iwork + 5 * mk) + j : lpiv;
#define dl(i) dlp[(i) * sw]
#define dg(i) dgp[(i) * sw]
#define du(i) dup[(i) * sw]
#define du2(i) du2p[(i) * sw]
#define z(i) zp[(i) * sw]
#define piv(i) pivp[(i) * sw]
    for (int i = 0; i < M; ++i) {
      dg(i) = dd[i] - lam;
      dl(i) = (i < M - 1) ? ee[i] : 0.0;
      du(i) = (i < M - 1) ? ee[i] : 0.0;
      du2(i) = 0.0;
    }
    const double tiny = 1e-15 * fmax(tnorm, 1e-300);
    for (int i = 0; i < M - 1; ++i) {
      if (fabs(dg(i)) >= fabs(dl(i))) {
        piv(i) = 0;
        if (dg(i) == 0.0) dg(i) = tiny;
        const double f = dl(i) / dg(i);
        dl(i) = f;
        dg(i + 1) -= f * du(i);
      } else {
        piv(i) = 1;
        const double f = dg(i) / dl(i);
        dg(i) = dl(i);
        dl(i) = f;
        const double tmp = du(i);
        du(i) = dg(i + 1);
        dg(i + 1) = tmp - f * dg(i + 1);
        if (i < M - 2) {
          du2(i) = du(i + 1);
          du(i + 1) = -f * du(i + 1);
        }
      }
    }
    if (dg(M - 1) == 0.0) dg(M - 1) = tiny;
    for (int i = 0; i < M; ++i) dg(i) = 1.0 / dg(i);  // reciprocal pivots: the solves multiply
    unsigned h = 2166136261u ^ (unsigned)(j * 16777619u);
    for (int i = 0; i < M; ++i) {
      h = h * 1664525u + 1013904223u;
      z(i) = ((h >> 8) * (1.0 / 16777216.0)) - 0.5;
    }
    for (int rep = 0; rep < 3; ++rep) {
      for (int i = 0; i < M - 1; ++i) {
        if (piv(i) == 0) {
          z(i + 1) -= dl(i) * z(i);
        } else {
          const double tmp = z(i);
          z(i) = z(i + 1);
          z(i + 1) = tmp - dl(i) * z(i);
        }
      }
      z(M - 1) *= dg(M - 1);
      if (M > 1) z(M - 2) = (z(M - 2) - du(M - 2) * z(M - 1)) * dg(M - 2);
      for (int i = M - 3; i >= 0; --i) z(i) = (z(i) - du(i) * z(i + 1) - du2(i) * z(i + 2)) * dg(i);
      double nrm = 0.0;
      for (int i = 0; i < M; ++i) nrm = fmax(nrm, fabs(z(i)));
      const double inv = nrm > 0.0 ? 1.0 / nrm : 1.0;
      for (int i = 0; i < M; ++i) z(i) *= inv;
    }
    double n2 = 0.0;
    for (int i = 0; i < M; ++i) n2 += z(i) * z(i);
    const double inv = 1.0 / sqrt(n2);
    for (int i = 0; i < M; ++i) Z[i * Kp + j] = z(i) * inv;
#undef dl
#undef dg
#undef du
#undef du2
#undef z
#undef piv
  }
  __syncthreads();
  // Gram-Schmidt inside clusters only (as LAPACK's inverse iteration does):
  // eigenvalues closer than 1e-3 |T| to their neighbour form a cluster, and
  // a vector is orthogonalised, twice, against the earlier vectors of its
  // cluster, then normalised.  Vectors of separated eigenvalues are already
  // orthogonal to ~eps |T| / gap.  Every thread derives the same clusters
  // from theta, so the barriers below are uniform.
  const double ortol = 1e-3 * fmax(tnorm, 1e-300);
  int cs = 0;  // first vector of the current cluster
  for (int j = 0; j < Kp; ++j) {
    if (j > 0 && theta[j] - theta[j - 1] > ortol) cs = j;
    if (cs == j) continue;
    for (int pass = 0; pass < 2; ++pass) {
      for (int i = cs + warp; i < j; i += nwarp) {
        double dt = 0.0;
        for (int r = lane; r < M; r += 32) dt += Z[r * Kp + i] * Z[r * Kp + j];
        dt = warp_sum(dt);
        if (lane == 0) red[i] = dt;
      }
      __syncthreads();
      for (int r = tid; r < M; r += nt) {
        double vz = Z[r * Kp + j];
        for (int i = cs; i < j; ++i) vz -= red[i] * Z[r * Kp + i];
        Z[r * Kp + j] = vz;
      }
      __syncthreads();
    }
    if (warp == 0) {
      double n2 = 0.0;
      for (int r = lane; r < M; r += 32) n2 += Z[r * Kp + j] * Z[r * Kp + j];
      n2 = warp_sum(n2);
      if (lane == 0) red[kKeepMax] = 1.0 / sqrt(n2);
    }
    __syncthreads();
    const double inv = red[kKeepMax];
    for (int r = tid; r < M; r += nt) Z[r * Kp + j] *= inv;
    __syncthreads();
  }
  // ---- 4. back-transformation: S = H_0 H_1 ... H_{M-2} Z ----
  // Reflectors in blocks of nbw, the last block first.  A block's product is
  // H_k0 ... H_k1-1 = I - V T V^H with T^-1 = diag(1/tau) + strict_upper(V^H V)
  // (the "UT transform" of compact WY), so S <- S - V T (V^H S) needs only the
  // block's Gram matrix G = V^H V: Y = V^H S, then T Y by back-substitution,
  // Y'_c = tau_c (Y_c - sum_{b > c} G_cb Y'_b) (tau_c = 0 gives 0, as it must),
  // then S -= V Y'.  G and Y live in Z's space (kJacobiMax x kKeepMax doubles
  // in every caller), free once S holds Z; nbw is the largest block (<= 16)
  // that fits there.
  for (int i = tid; i < M * Kp; i += nt) S[i] = make_double2(Z[i], 0.0);
  __syncthreads();
  int nbw = 16;
  while (nbw > 1 && 2 * nbw * (nbw + Kp) > kJacobiMax * kKeepMax) --nbw;
  double2* Gv = reinterpret_cast<double2*>(Z);  // nbw x nbw, strict upper part
  double2* Yv = Gv + nbw * nbw;                 // nbw x Kp
  for (int k1 = M - 1; k1 > 0; k1 -= nbw) {     // reflectors k0 .. k1-1
    const int k0 = max(0, k1 - nbw);
    const int nb = k1 - k0;
    // v_c (reflector k = k0 + c) at row r: 0 for r <= k, 1 at r = k + 1, A[r][k] below.
    // One thread per output entry, a serial dot over the rows: G[a][c] =
    // v_a^H v_c (a < c) for the first nb*nb entries, Y[c][j] = v_c^H s_j after
    for (int e = tid; e < nb * nb + nb * Kp; e += nt) {
      double2 acc = make_double2(0.0, 0.0);
      if (e < nb * nb) {
        const int ga = e / nb, gc = e % nb;
        if (ga >= gc) continue;
        const int ka = k0 + ga, kc = k0 + gc;
        acc = cconj(A[(kc + 1) * lda + ka]);  // v_c's unit entry; v_a there and below is A[r][ka]
        for (int r = kc + 2; r < M; ++r) acc = cadd(acc, cdotc(A[r * lda + ka], A[r * lda + kc]));
        Gv[ga * nbw + gc] = acc;
      } else {
        const int f = e - nb * nb;
        const int c = f / Kp, j = f % Kp;
        const int k = k0 + c;
        acc = S[(k + 1) * Kp + j];
        for (int r = k + 2; r < M; ++r) acc = cadd(acc, cdotc(A[r * lda + k], S[r * Kp + j]));
        Yv[f] = acc;
      }
    }
    __syncthreads();
    // Y <- T Y by back-substitution, one thread per column j (rows descending)
    for (int j = tid; j < Kp; j += nt) {
      for (int c = nb - 1; c >= 0; --c) {
        double2 acc = Yv[c * Kp + j];
        for (int bb = c + 1; bb < nb; ++bb) acc = csub(acc, cmul(Gv[c * nbw + bb], Yv[bb * Kp + j]));
        Yv[c * Kp + j] = cmul(tau[k0 + c], acc);
      }
    }
    __syncthreads();
    // S -= V Y on rows k0+1 .. M-1
    for (int e = tid; e < (M - k0 - 1) * Kp; e += nt) {
      const int r = k0 + 1 + e / Kp, j = e % Kp;
      double2 acc = make_double2(0.0, 0.0);
      for (int c = 0; c < nb; ++c) {
        const int k = k0 + c;
        if (r <= k) break;
        const double2 vr = (r == k + 1) ? make_double2(1.0, 0.0) : A[r * lda + k];
        acc = cadd(acc, cmul(vr, Yv[c * Kp + j]));
      }
      S[r * Kp + j] = csub(S[r * Kp + j], acc);
    }
    __syncthreads();
  }
  __syncthreads();
}

// Ritz step: per instance, when due.  Dynamic smem: 2 * kJacobiMax^2 double2.
constexpr int kRitzThreads = 256;  // one CTA per instance (512 measured no faster: serial FP64 chains)
__global__ void __launch_bounds__(kRitzThreads) k_lz_ritz(rsed_lanczos_t st, LzDims d, int check_every, int force,
                                                         int rr) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int inst = blockIdx.x;
  int* stt = st.state + inst * kStateInts;
  if (rr) {
    if (stt[S_RR] != 1) return;
  } else if (!stt[S_ACTIVE]) {
    return;
  }
  const int b = st.inst_b[inst];
  const int nb = rr ? st.keep_blocks + 2 : stt[S_NB];
  const int M = (nb - 1) * b;
  const bool full = !rr && (nb >= d.n_slots + 1);
  const int nev = st.nev;
  const int K = st.keep_blocks * b;
  const bool due = rr || full || force || (M >= nev + b && M >= K && (stt[S_ITERS] % check_every) == 0);
  if (!due) return;
  if (M < nev || M < K || M > kJacobiMax) {
    if (full && threadIdx.x == 0) {  // cannot restart: report instead of overrunning
      stt[S_STATUS] = RSED_EINVAL;
      stt[S_ACTIVE] = 0;
    }
    return;
  }
  double2* A = reinterpret_cast<double2*>(smem);
  double2* Sv = A + kJacobiMax * (kJacobiMax + 1);                // M x Kp eigenvectors
  double* Z = reinterpret_cast<double*>(Sv + kJacobiMax * kKeepMax);  // M x Kp real scratch
  __shared__ double2 tau[kJacobiMax], vv[kJacobiMax], pw[kJacobiMax];
  __shared__ double dd[kJacobiMax], ee[kJacobiMax], red[64];
  __shared__ double theta[kKeepMax];
  __shared__ int conv_flag;
  const int Kp = min(M, max(nev, K));
  const double2* P = reinterpret_cast<const double2*>(st.P) + (int64_t)inst * d.pm * d.pm;
  for (int i = threadIdx.x; i < M * M; i += blockDim.x) {
    const int r = i / M, c = i % M;
    const double2 a = P[(int64_t)r * d.pm + c], bt = P[(int64_t)c * d.pm + r];
    A[r * (M + 1) + c] = make_double2(0.5 * (a.x + bt.x), 0.5 * (a.y - bt.y));
  }
  __syncthreads();
  herm_lowest(A, M, Kp, theta, Sv, Z, tau, dd, ee, red, vv, pw,
              reinterpret_cast<double*>(Z + kJacobiMax * kKeepMax));
  double* rv = st.ritz_val + (int64_t)inst * d.pm;
  double2* rvec = reinterpret_cast<double2*>(st.ritz_vec) + (int64_t)inst * d.pm * d.pm;
  double* res = st.resid + (int64_t)inst * d.pm;
  for (int i = threadIdx.x; i < M * Kp; i += blockDim.x) {
    const int r = i / Kp, j = i % Kp;
    rvec[(int64_t)r * d.pm + j] = Sv[r * Kp + j];
  }
  for (int j = threadIdx.x; j < Kp; j += blockDim.x) rv[j] = theta[j];
  __syncthreads();
  if (rr) {  // Rayleigh-Ritz refinement: eigenpairs only, residuals come from k_rr_resid
    if (threadIdx.x == 0) {
      stt[S_NB] = nb;
      stt[S_RR] = 2;
    }
    return;
  }
  // residual estimates: || Rlast * S[last block rows, j] ||
  for (int j = threadIdx.x; j < Kp; j += blockDim.x) {
    double acc = 0.0;
    for (int q = 0; q < b; ++q) {
      double2 v = make_double2(0.0, 0.0);
      for (int p = 0; p < b; ++p) {
        const double2 r = P[(int64_t)((nb - 1) * b + q) * d.pm + (nb - 2) * b + p];
        v = cadd(v, cmul(r, Sv[((nb - 2) * b + p) * Kp + j]));
      }
      acc += v.x * v.x + v.y * v.y;
    }
    res[j] = sqrt(acc);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int nconv = 0;
    for (int j = 0; j < nev; ++j) {
      if (res[j] <= st.tol * fmax(1.0, fabs(rv[j]))) ++nconv;
      else break;
    }
    stt[S_NCONV] = nconv;
    conv_flag = (nconv >= nev);
    if (conv_flag) {
      stt[S_STATUS] = 1;
      stt[S_ACTIVE] = 0;
    } else if (full) {
      stt[S_RESTARTS] += 1;
      if (stt[S_RESTARTS] > st.max_restarts) {
        stt[S_STATUS] = RSED_ENOTCONV;
        stt[S_ACTIVE] = 0;
        conv_flag = 1;  // no restart
      }
    }
  }
  __syncthreads();
  if (conv_flag || !full) return;
  // thick restart: new projected matrix diag(theta_0..K-1) + coupling block
  double2* Pw = reinterpret_cast<double2*>(st.P) + (int64_t)inst * d.pm * d.pm;
  // coupling rows first (needs old P), staged in smem A (free now)
  for (int it = threadIdx.x; it < b * K; it += blockDim.x) {
    const int q = it / K, j = it % K;
    double2 v = make_double2(0.0, 0.0);
    for (int p = 0; p < b; ++p) {
      const double2 r = Pw[(int64_t)((nb - 1) * b + q) * d.pm + (nb - 2) * b + p];
      v = cadd(v, cmul(r, Sv[((nb - 2) * b + p) * Kp + j]));
    }
    A[it] = v;
  }
  __syncthreads();
  const int Mn = (st.keep_blocks + 1) * b;
  for (int i = threadIdx.x; i < (nb)*b * (nb)*b; i += blockDim.x) {
    const int r = i / (nb * b), c = i % (nb * b);
    Pw[(int64_t)r * d.pm + c] = make_double2(0.0, 0.0);
  }
  __syncthreads();
  for (int j = threadIdx.x; j < K; j += blockDim.x) Pw[(int64_t)j * d.pm + j] = make_double2(rv[j], 0.0);
  for (int it = threadIdx.x; it < b * K; it += blockDim.x) {
    const int q = it / K, j = it % K;
    Pw[(int64_t)(K + q) * d.pm + j] = A[it];
  }
  (void)Mn;
  if (threadIdx.x == 0) {
    stt[S_RESTART_NB] = nb;
    stt[S_NB] = st.keep_blocks + 1;
  }
}

// V_0..keep-1 = V S_keep ; residual block (old slot nb_old-1) -> slot keep.
// Block (row range, instance) with the instance's Ritz coefficients staged in
// shared memory; one row per thread.
__global__ void __launch_bounds__(256) k_lz_restart(rsed_lanczos_t st, LzDims d) {
  const int inst = blockIdx.x % d.n_inst;  // instances of one row range adjacent in launch order
  const int64_t rblock = blockIdx.x / d.n_inst;
  const int* stt = st.state + inst * kStateInts;
  const int nb_old = stt[S_RESTART_NB];
  if (nb_old == 0) return;
  const int b = st.inst_b[inst];
  const int c0 = st.inst_col0[inst];
  const int K = st.keep_blocks * b;
  const int Mold = (nb_old - 1) * b;
  if (Mold > kJacobiMax || K > kKeepMax) return;
  __shared__ double2 Ss[kJacobiMax * kKeepMax];
  const double2* S = reinterpret_cast<const double2*>(st.ritz_vec) + (int64_t)inst * d.pm * d.pm;
  for (int e = threadIdx.x; e < Mold * K; e += blockDim.x) Ss[(e / K) * kKeepMax + e % K] = S[(int64_t)(e / K) * d.pm + e % K];
  __syncthreads();
  const int64_t row = rblock * blockDim.x + threadIdx.x;
  if (row >= d.n_orb) return;
  double2* V = reinterpret_cast<double2*>(st.V);
  const int64_t slot_stride = d.n_orb * d.ld;
  double2 acc[kKeepMax];
#pragma unroll
  for (int j = 0; j < kKeepMax; ++j) acc[j] = make_double2(0.0, 0.0);
#pragma unroll 8
  for (int l = 0; l < Mold; ++l) {
    const double2 v = V[(int64_t)(l / b) * slot_stride + row * d.ld + c0 + (l % b)];
#pragma unroll
    for (int j = 0; j < kKeepMax; ++j)
      if (j < K) acc[j] = cadd(acc[j], cmul(v, Ss[l * kKeepMax + j]));
  }
  double2 resid[kBMax];
#pragma unroll
  for (int q = 0; q < kBMax; ++q)
    if (q < b) resid[q] = V[(int64_t)(nb_old - 1) * slot_stride + row * d.ld + c0 + q];
#pragma unroll
  for (int j = 0; j < kKeepMax; ++j)
    if (j < K) V[(int64_t)(j / b) * slot_stride + row * d.ld + c0 + (j % b)] = acc[j];
#pragma unroll
  for (int q = 0; q < kBMax; ++q)
    if (q < b) V[(int64_t)st.keep_blocks * slot_stride + row * d.ld + c0 + q] = resid[q];
}

// The same restart for all instances at once: thread = (row, column c0 + q)
// of RG row groups per grid-stride iteration, so every basis slot is read
// as whole contiguous rows.  The Ritz coefficients of all restarting
// instances sit in shared memory column-major,
//   St[((l*bmax + p)*keep + jb)*ld + c0 + q] = S_i[l*b + p][jb*b + q],
// so the lanes of a warp read consecutive words.  Every thread of the block
// finishes reading its two rows (block barrier) before the rows are
// overwritten in place.  KM bounds keep_blocks (register accumulators), BB
// the block size; each coefficient read from shared memory serves the RG rows.
template <int KM, int RG, int BB>
__global__ void __launch_bounds__(256, 2) k_lz_restart_rows(rsed_lanczos_t st, LzDims d) {
  extern __shared__ __align__(16) unsigned char smem_r[];
  const int keep = st.keep_blocks, bmax = st.bmax, ld = d.ld;
  double2* St = reinterpret_cast<double2*>(smem_r);
  int* meta = reinterpret_cast<int*>(St + (size_t)d.n_slots * bmax * keep * ld);  // [ld]
  for (int c = threadIdx.x; c < ld; c += blockDim.x) meta[c] = -1;
  __syncthreads();
  for (int inst = threadIdx.x; inst < d.n_inst; inst += blockDim.x) {
    const int nb_old = st.state[inst * kStateInts + S_RESTART_NB];
    const int b = st.inst_b[inst], c0 = st.inst_col0[inst];
    // a restart comes when the basis holds n_slots + 1 blocks (the last in the spare slot)
    if (nb_old < 1 || nb_old > d.n_slots + 1 || (nb_old - 1) * b > kJacobiMax || keep * b > kKeepMax) continue;
    for (int q = 0; q < b; ++q) meta[c0 + q] = inst;
  }
  __syncthreads();
  for (int inst = 0; inst < d.n_inst; ++inst) {
    const int b = st.inst_b[inst], c0 = st.inst_col0[inst];
    if (meta[c0] != inst) continue;
    const int nb_old = st.state[inst * kStateInts + S_RESTART_NB];
    const int Mold = (nb_old - 1) * b, K = keep * b;
    const double2* S = reinterpret_cast<const double2*>(st.ritz_vec) + (int64_t)inst * d.pm * d.pm;
    for (int e = threadIdx.x; e < Mold * K; e += blockDim.x) {
      const int l = e / K, j = e % K;
      St[((size_t)((l / b) * bmax + l % b) * keep + j / b) * ld + c0 + j % b] = S[(int64_t)l * d.pm + j];
    }
  }
  __syncthreads();
  const int rows_pg = blockDim.x / ld;
  const int rloc = threadIdx.x / ld, col = threadIdx.x % ld;
  const int inst = rloc < rows_pg ? meta[col] : -1;
  int b = 1, c0 = 0, nslot = 0;
  if (inst >= 0) {
    b = st.inst_b[inst];
    c0 = st.inst_col0[inst];
    nslot = st.state[inst * kStateInts + S_RESTART_NB] - 1;  // basis blocks combined
  }
  double2* V = reinterpret_cast<double2*>(st.V);
  const int64_t slot_stride = d.n_orb * d.ld;
  const int64_t n_groups = (d.n_orb + rows_pg - 1) / rows_pg;
  const double2* scol = St + col;
  const int64_t gstride = (int64_t)rows_pg * ld;  // one row group further
  for (int64_t grp = RG * (int64_t)blockIdx.x; grp < n_groups; grp += RG * (int64_t)gridDim.x) {
    const int64_t row0 = grp * rows_pg + rloc;
    bool live[RG];
    double2 a[RG][KM], r[RG];
#pragma unroll
    for (int h = 0; h < RG; ++h) {
      live[h] = inst >= 0 && row0 + h * rows_pg < d.n_orb;
      r[h] = make_double2(0.0, 0.0);
#pragma unroll
      for (int j = 0; j < KM; ++j) a[h][j] = make_double2(0.0, 0.0);
    }
    if (live[0]) {
#pragma unroll 2
      for (int l = 0; l < nslot; ++l) {
        const double2* Vs = V + (int64_t)l * slot_stride + row0 * ld + c0;
#pragma unroll
        for (int p = 0; p < BB; ++p) {
          if (p >= b) break;
          double2 v[RG];
#pragma unroll
          for (int h = 0; h < RG; ++h) v[h] = live[h] ? Vs[h * gstride + p] : make_double2(0.0, 0.0);
          const double2* sp = scol + (size_t)((l * bmax + p) * keep) * ld;
#pragma unroll
          for (int j = 0; j < KM; ++j) {
            if (j < keep) {
              const double2 c = sp[(size_t)j * ld];
#pragma unroll
              for (int h = 0; h < RG; ++h) a[h][j] = cadd(a[h][j], cmul(v[h], c));
            }
          }
        }
      }
#pragma unroll
      for (int h = 0; h < RG; ++h)
        if (live[h]) r[h] = V[(int64_t)nslot * slot_stride + row0 * ld + h * gstride + col];
    }
    __syncthreads();  // the rows of these groups are read by every thread before any is overwritten
#pragma unroll
    for (int h = 0; h < RG; ++h) {
      if (!live[h]) continue;
      const int64_t at = row0 * ld + h * gstride + col;
#pragma unroll
      for (int j = 0; j < KM; ++j)
        if (j < keep) V[(int64_t)j * slot_stride + at] = a[h][j];
      V[(int64_t)keep * slot_stride + at] = r[h];
    }
  }
}

// U[inst][j][row] = sum_l V_l[row] S[l][j], j < nev (Ritz vectors of the last check).
__global__ void __launch_bounds__(256) k_lz_extract(rsed_lanczos_t st, LzDims d, double2* U, int64_t u_stride) {
  const int inst = blockIdx.x % d.n_inst;
  const int64_t rblock = blockIdx.x / d.n_inst;
  const int* stt = st.state + inst * kStateInts;
  const int b = st.inst_b[inst];
  const int c0 = st.inst_col0[inst];
  const int nb = stt[S_NB];
  const int M = (nb - 1) * b;
  const int nev = st.nev;
  if (M > kJacobiMax + kBMax || nev > kKeepMax) return;
  __shared__ double2 Ss[(kJacobiMax + kBMax) * kKeepMax];
  const double2* S = reinterpret_cast<const double2*>(st.ritz_vec) + (int64_t)inst * d.pm * d.pm;
  for (int e = threadIdx.x; e < M * nev; e += blockDim.x)
    Ss[(e / nev) * kKeepMax + e % nev] = S[(int64_t)(e / nev) * d.pm + e % nev];
  __syncthreads();
  const int64_t row = rblock * blockDim.x + threadIdx.x;
  if (row >= d.n_orb) return;
  const double2* V = reinterpret_cast<const double2*>(st.V);
  const int64_t slot_stride = d.n_orb * d.ld;
  double2 acc[kKeepMax];
#pragma unroll
  for (int j = 0; j < kKeepMax; ++j) acc[j] = make_double2(0.0, 0.0);
  for (int l = 0; l < M; ++l) {
    const double2 v = V[(int64_t)(l / b) * slot_stride + row * d.ld + c0 + (l % b)];
#pragma unroll
    for (int j = 0; j < kKeepMax; ++j)
      if (j < nev) acc[j] = cadd(acc[j], cmul(v, Ss[l * kKeepMax + j]));
  }
#pragma unroll
  for (int j = 0; j < kKeepMax; ++j)
    if (j < nev) U[((int64_t)inst * nev + j) * u_stride + row] = acc[j];
}

// ---------------------------------------------------------------------------
// FP64 Rayleigh-Ritz refinement of a converged (FP32-matvec) solve.
// k_rr_prepare flags converged instances and schedules the thick-restart
// combination (V_0..keep-1 = Ritz vectors, residual block -> slot keep);
// the caller then applies H in FP64 to slots 0..keep (into slots keep+1..),
// k_rr_gram forms T = Q^H H Q over those K + b vectors, k_lz_ritz(rr)
// diagonalises its Hermitian part and k_rr_resid measures the true FP64
// residuals ||H u_j - theta_j u_j||.
__global__ void k_rr_prepare(rsed_lanczos_t st) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= st.n_inst) return;
  int* s = st.state + i * kStateInts;
  if (s[S_STATUS] == 1 && s[S_RR] == 0) {
    s[S_RESTART_NB] = s[S_NB];
    s[S_NB] = st.keep_blocks + 1;
    s[S_RR] = 1;
  }
}

// Each task (row r of T, column block l2) is split over NP = blockDim / tasks
// row phases (interleaved rows), summed in phase order in shared memory.
__global__ void __launch_bounds__(256) k_rr_gram(rsed_lanczos_t st, LzDims d) {
  const int chunk = blockIdx.x / d.n_inst;
  const int inst = blockIdx.x % d.n_inst;
  int* stt = st.state + inst * kStateInts;
  if (stt[S_RR] != 1) return;
  const int b = st.inst_b[inst];
  const int c0 = st.inst_col0[inst];
  const int nq = st.keep_blocks + 1;  // blocks of Q
  const int M = nq * b;
  const int64_t r0 = (int64_t)chunk * d.chunk_rows;
  const int64_t r1 = min(r0 + d.chunk_rows, d.n_orb);
  const double2* V = reinterpret_cast<const double2*>(st.V);
  const int64_t slot_stride = d.n_orb * d.ld;
  double2* part = reinterpret_cast<double2*>(st.partial);
  const int64_t pbase = ((int64_t)chunk * d.n_inst + inst) * (int64_t)kRRMax * kRRMax;
  __shared__ int s_last;
  // thread task: (row of T, column block l2, row phase) -> b accumulators
  __shared__ double2 red[256][kBMax];
  const int n_tasks = M * nq;
  const int NP = n_tasks >= (int)blockDim.x ? 1 : (int)blockDim.x / n_tasks;
  for (int t0 = 0; t0 < n_tasks * NP; t0 += blockDim.x) {  // one pass when NP > 1
    const int t = t0 + (int)threadIdx.x;
    const bool act = t < n_tasks * NP;
    const int task = t % n_tasks, ph = t / n_tasks;
    const int r = task / nq, l2 = task % nq;
    double2 acc[kBMax];
#pragma unroll
    for (int q = 0; q < kBMax; ++q) acc[q] = make_double2(0.0, 0.0);
    if (act) {
      const double2* Q = V + (int64_t)(r / b) * slot_stride + c0 + (r % b);
      const double2* Z = V + (int64_t)(nq + l2) * slot_stride + c0;
#pragma unroll 4
      for (int64_t row = r0 + ph; row < r1; row += NP) {
        const double2 qv = Q[row * d.ld];
#pragma unroll
        for (int q = 0; q < kBMax; ++q)
          if (q < b) acc[q] = cadd(acc[q], cdotc(qv, Z[row * d.ld + q]));
      }
    }
    if (NP == 1) {
      if (act) {
#pragma unroll
        for (int q = 0; q < kBMax; ++q)
          if (q < b) part[pbase + r * kRRMax + l2 * b + q] = acc[q];
      }
    } else {
#pragma unroll
      for (int q = 0; q < kBMax; ++q) red[threadIdx.x][q] = acc[q];
      __syncthreads();
      if ((int)threadIdx.x < n_tasks) {
#pragma unroll
        for (int q = 0; q < kBMax; ++q) {
          if (q >= b) continue;
          double2 a = make_double2(0.0, 0.0);
          for (int h = 0; h < NP; ++h) a = cadd(a, red[threadIdx.x + h * n_tasks][q]);
          part[pbase + r * kRRMax + l2 * b + q] = a;
        }
      }
      __syncthreads();
    }
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const int t = atomicAdd(&stt[S_TICKET], 1);
    s_last = (t == d.n_chunks - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (threadIdx.x == 0) {
    stt[S_TICKET] = 0;
    stt[S_RESTART_NB] = 0;
  }
  double2* P = reinterpret_cast<double2*>(st.P) + (int64_t)inst * d.pm * d.pm;
  // G threads per entry over interleaved chunk subsets, then in order
  __shared__ double2 fin[kRRMax * kRRMax];
  const int nent = M * M;
  const int G = max(1, (int)blockDim.x / nent);
  for (int t = threadIdx.x; t < nent * G; t += blockDim.x) {
    const int e = t % nent, g = t / nent, r = e / M, c = e % M;
    double2 a = make_double2(0.0, 0.0);
#pragma unroll 8
    for (int ch = g; ch < d.n_chunks; ch += G)
      a = cadd(a, __ldcg(part + ((int64_t)ch * d.n_inst + inst) * (int64_t)kRRMax * kRRMax + r * kRRMax + c));
    fin[g * nent + e] = a;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nent; e += blockDim.x) {
    double2 a = make_double2(0.0, 0.0);
    for (int g = 0; g < G; ++g) a = cadd(a, fin[g * nent + e]);
    P[(int64_t)(e / M) * d.pm + e % M] = a;
  }
}

// True FP64 residual norms of the nev refined pairs.
__global__ void __launch_bounds__(128) k_rr_resid(rsed_lanczos_t st, LzDims d) {
  const int chunk = blockIdx.x / d.n_inst;
  const int inst = blockIdx.x % d.n_inst;
  int* stt = st.state + inst * kStateInts;
  if (stt[S_RR] != 2) return;
  const int b = st.inst_b[inst];
  const int c0 = st.inst_col0[inst];
  const int nq = st.keep_blocks + 1;
  const int M = nq * b;
  const int nev = st.nev;
  const int64_t r0 = (int64_t)chunk * d.chunk_rows;
  const int64_t r1 = min(r0 + d.chunk_rows, d.n_orb);
  const double2* V = reinterpret_cast<const double2*>(st.V);
  const int64_t slot_stride = d.n_orb * d.ld;
  const double2* S = reinterpret_cast<const double2*>(st.ritz_vec) + (int64_t)inst * d.pm * d.pm;
  const double* th = st.ritz_val + (int64_t)inst * d.pm;
  double* part = st.partial;
  __shared__ double red[kKeepMax][128];
  __shared__ int s_last;
  for (int j = 0; j < nev; ++j) red[j][threadIdx.x] = 0.0;
  for (int64_t row = r0 + threadIdx.x; row < r1; row += blockDim.x) {
    for (int j = 0; j < nev; ++j) {
      double2 hu = make_double2(0.0, 0.0), u = make_double2(0.0, 0.0);
      for (int l = 0; l < M; ++l) {
        const double2 sj = S[(int64_t)l * d.pm + j];
        const int64_t off = row * d.ld + c0 + (l % b);
        u = cadd(u, cmul(V[(int64_t)(l / b) * slot_stride + off], sj));
        hu = cadd(hu, cmul(V[(int64_t)(nq + l / b) * slot_stride + off], sj));
      }
      const double2 r = make_double2(hu.x - th[j] * u.x, hu.y - th[j] * u.y);
      red[j][threadIdx.x] += r.x * r.x + r.y * r.y;
    }
  }
  __syncthreads();
  for (int w = 64; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int j = 0; j < nev; ++j) red[j][threadIdx.x] += red[j][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < nev)
    part[((int64_t)chunk * d.n_inst + inst) * kKeepMax + threadIdx.x] = red[threadIdx.x][0];
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const int t = atomicAdd(&stt[S_TICKET], 1);
    s_last = (t == d.n_chunks - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (threadIdx.x == 0) stt[S_TICKET] = 0;
  if (threadIdx.x < nev) {
    double a = 0.0;
    for (int ch = 0; ch < d.n_chunks; ++ch)
      a += __ldcg(part + ((int64_t)ch * d.n_inst + inst) * kKeepMax + threadIdx.x);
    st.resid[(int64_t)inst * d.pm + threadIdx.x] = sqrt(a);
  }
  if (threadIdx.x == 0) stt[S_RR] = 3;
}

// ---------------------------------------------------------------------------
// Persistent form: one thread-block cluster per instance runs the whole
// thick-restart loop in one launch.  CTA r of the cluster owns a contiguous
// slice of the orbit rows; per iteration
//   matvec (own rows, x gathered from every row) -> Gram partials of own rows
//   -> cluster barrier -> CTA 0 sums the partials through distributed shared
//   memory, factors, updates P -> cluster barrier -> every CTA reads C, R
//   from CTA 0 and updates its rows -> (second pass likewise) -> at a full
//   basis CTA 0 solves the projected eigenproblem and every CTA recombines
//   its rows for the thick restart.
// Control values live in CTA 0's shared memory and are read by all CTAs after
// a cluster barrier, so every CTA takes the same branch and executes the same
// number of barriers.  Waiting is only on hardware cluster barriers; the loop
// is bounded by max_iter.
constexpr int kPT = 512;          // threads per CTA
constexpr int kHopLanes = 4;      // lanes sharing one row's hops in the matvec
constexpr int kPHB = 4;           // hops whose loads are issued together
constexpr int kPB = 4;            // largest block size of the persistent form
constexpr int kPRows = kJacobiMax + kBMax;  // max rows of the Gram matrices

struct PersistLayout {
  size_t part, tot, c1, c2, r1, r2, sg, sloc, eigA, eigS, eigZ, total;
};

enum { C_NB = 0, C_ACTIVE, C_ITERS, C_RESTARTS, C_STATUS, C_OK, C_RESTART, C_NBOLD, C_NCONV, C_N };

template <int PREC>
__global__ void __launch_bounds__(kPT, 1)
k_lz_persist(rsed_model_t md, rsed_sectors_t sc, rsed_lanczos_t st, LzDims d, rsed_apply::ApplySmemLayout alay,
             PersistLayout pl, int max_iter) {
  using XT = typename std::conditional<PREC == 64, double2, float2>::type;
  cg::cluster_group cluster = cg::this_cluster();
  const int CS = (int)cluster.num_blocks();
  const int rank = (int)cluster.block_rank();
  const int inst = blockIdx.x / CS;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = kPT >> 5;
  extern __shared__ __align__(16) unsigned char smem[];
  rsed_apply::ApplyView av = rsed_apply::stage_apply(md, sc, alay, smem);
  double2* part = reinterpret_cast<double2*>(smem + pl.part);  // [kPRows][kBMax]
  double2* tot = reinterpret_cast<double2*>(smem + pl.tot);
  double2* C1 = reinterpret_cast<double2*>(smem + pl.c1);
  double2* C2 = reinterpret_cast<double2*>(smem + pl.c2);
  double2* R1 = reinterpret_cast<double2*>(smem + pl.r1);     // [kBMax][kBMax]
  double2* R2 = reinterpret_cast<double2*>(smem + pl.r2);
  double2* sG = reinterpret_cast<double2*>(smem + pl.sg);
  double2* Sloc = reinterpret_cast<double2*>(smem + pl.sloc);  // [kJacobiMax][kKeepMax]
  __shared__ int ctl[C_N];
  __shared__ double2 tau[kJacobiMax], vv[kJacobiMax], pw[kJacobiMax];
  __shared__ double dd[kJacobiMax], ee[kJacobiMax], red[64], theta[kKeepMax], resj[kKeepMax];

  int* stt = st.state + inst * kStateInts;
  const int b = st.inst_b[inst];
  const int c0 = st.inst_col0[inst];
  const int sector = av.csec[c0];
  const int nev = st.nev, keep = st.keep_blocks, K = keep * b;
  const int64_t slot = d.n_orb * d.ld;
  const int64_t per = (d.n_orb + CS - 1) / CS;
  const int64_t rb = (int64_t)rank * per, re = min(rb + per, d.n_orb);
  double2* V = reinterpret_cast<double2*>(st.V);
  double2* W = reinterpret_cast<double2*>(st.W);
  double2* X = V + (int64_t)(d.n_slots + 1) * slot;
  const XT* xin = (PREC == 64) ? reinterpret_cast<const XT*>(X) : reinterpret_cast<const XT*>(st.Xf);
  double2* P = reinterpret_cast<double2*>(st.P) + (int64_t)inst * d.pm * d.pm;
  const int kp1 = md.n_filled + 1;
  const bool bad_block = (b < 1 || b > kPB || (32 % b) != 0);

  if (rank == 0 && tid == 0) {
    ctl[C_NB] = stt[S_NB];
    ctl[C_ACTIVE] = stt[S_ACTIVE] && !bad_block;
    ctl[C_ITERS] = stt[S_ITERS];
    ctl[C_RESTARTS] = stt[S_RESTARTS];
    ctl[C_STATUS] = bad_block ? RSED_EINVAL : stt[S_STATUS];
    ctl[C_OK] = 1;
    ctl[C_RESTART] = 0;
    ctl[C_NBOLD] = 0;
    ctl[C_NCONV] = stt[S_NCONV];
  }
  int* ctl0 = cluster.map_shared_rank(ctl, 0);

  for (int it = 0; it < max_iter; ++it) {
    cluster.sync();  // (A) X complete, control stable
    const int nb = ctl0[C_NB];
    if (!ctl0[C_ACTIVE]) break;
    // C_RESTART is next read after barrier (C) of this iteration's second pass
    if (rank == 0 && tid == 0) ctl[C_RESTART] = 0;
    // ---- matvec: W = H^dagger X on own rows (own columns) ----
    {
      const int ng = kPT / kHopLanes;
      const int hl = tid % kHopLanes;
      for (int64_t r0 = rb; r0 < re; r0 += ng) {
        const int64_t row = r0 + tid / kHopLanes;
        double2 acc[kPB];
#pragma unroll
        for (int q = 0; q < kPB; ++q) acc[q] = make_double2(0.0, 0.0);
        bool on = false;
        if (row < re) {
          const uint64_t memr = sc.member[row];
          on = (memr >> sector) & 1ull;
          if (on) {
            const uint64_t m = md.repr_masks[row];
            const double sr = sc.sqrt_stab[row];
            if (hl == 0) {
              const double2 hd = reinterpret_cast<const double2*>(md.hdiag)[row];
              for (int q = 0; q < b; ++q) {
                const XT xv = xin[row * d.ld + c0 + q];
                const double2 xx = make_double2((double)xv.x, (double)xv.y);
                acc[q] = cadd(acc[q], make_double2(hd.x * xx.x + hd.y * xx.y, hd.x * xx.y - hd.y * xx.x));
              }
            }
            int hop = 0;
            int bt[kPHB];
            int64_t bidx[kPHB];
            int nh = 0;
            auto process = [&](int cnt) {
              RsedEntry e[kPHB];
#pragma unroll
              for (int h = 0; h < kPHB; ++h)
                if (h < cnt) e[h] = rsed_apply::load_entry(reinterpret_cast<const RsedEntry*>(md.table), bidx[h]);
              uint64_t mc[kPHB];
              double sq[kPHB];
              XT xv[kPHB][kPB];
#pragma unroll
              for (int h = 0; h < kPHB; ++h) {
                if (h < cnt) {
                  const int64_t c = e[h].rep;
                  mc[h] = __ldg(sc.member + c);
                  sq[h] = __ldg(sc.sqrt_stab + c);
#pragma unroll
                  for (int q = 0; q < kPB; ++q)
                    if (q < b) xv[h][q] = xin[c * d.ld + c0 + q];
                }
              }
#pragma unroll
              for (int h = 0; h < kPHB; ++h) {
                if (h >= cnt || !((mc[h] >> sector) & 1ull)) continue;
                const int t = bt[h];
                double2 ta = cmul(av.tamp[t], make_double2(e[h].re, e[h].im));
                if (md.fermionic && (__popcll(m & av.tjw[t]) & 1)) {
                  ta.x = -ta.x;
                  ta.y = -ta.y;
                }
                const double ratio = sq[h] / sr;
                const double2 w =
                    cmul(make_double2(ta.x * ratio, -ta.y * ratio), av.chi[sector * md.n_group + e[h].g]);
#pragma unroll
                for (int q = 0; q < kPB; ++q) {
                  if (q < b) {
                    const double2 xx = make_double2((double)xv[h][q].x, (double)xv[h][q].y);
                    acc[q] = cadd(acc[q], cmul(w, xx));
                  }
                }
              }
            };
            uint64_t occ = m;
            while (occ) {
              const int i = __ffsll((long long)occ) - 1;
              occ &= occ - 1;
              const int t1 = av.tbeg[i + 1];
              for (int t = av.tbeg[i]; t < t1; ++t) {
                const int jj = av.tto[t];
                if ((m >> jj) & 1ull) continue;
                if ((hop++ % kHopLanes) != hl) continue;
                bt[nh] = t;
                bidx[nh] = rsed_rank_any(m ^ (1ull << i) ^ (1ull << jj), av.binom, kp1, md.species_b,
                                         md.species_b ? av.binom[__popcll(md.species_b) * kp1 + md.n_filled_b]
                                                      : 1);
                if (++nh == kPHB) {
                  process(kPHB);
                  nh = 0;
                }
              }
            }
            if (nh) process(nh);
          }
        }
#pragma unroll
        for (int q = 0; q < kPB; ++q) {
          for (int o = 1; o < kHopLanes; o <<= 1) {
            acc[q].x += __shfl_xor_sync(0xffffffffu, acc[q].x, o);
            acc[q].y += __shfl_xor_sync(0xffffffffu, acc[q].y, o);
          }
        }
        if (row < re && hl == 0)
          for (int q = 0; q < b; ++q) W[row * d.ld + c0 + q] = on ? acc[q] : make_double2(0.0, 0.0);
      }
    }
    __syncthreads();
    // ---- two Gram-Schmidt passes ----
    for (int pass = 1; pass <= 2; ++pass) {
      const int npairs = (nb + 1) * b;
      const int rl_n = 32 / b;           // row lanes per pair in a warp
      const int q = lane % b, rl = lane / b;
      for (int pair = warp; pair < npairs; pair += nwarp) {
        const int sl = pair / b, p = pair % b;
        const double2* Y = (sl < nb) ? V + sl * slot : W;
        double2 a = make_double2(0.0, 0.0);
        for (int64_t row = rb + rl; row < re; row += 4 * rl_n) {
          double2 yv[4], wv[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int64_t r = row + u * rl_n;
            yv[u] = (r < re) ? Y[r * d.ld + c0 + p] : make_double2(0.0, 0.0);
            wv[u] = (r < re) ? W[r * d.ld + c0 + q] : make_double2(0.0, 0.0);
          }
#pragma unroll
          for (int u = 0; u < 4; ++u) a = cadd(a, cdotc(yv[u], wv[u]));
        }
        for (int o = b; o < 32; o <<= 1) {
          a.x += __shfl_xor_sync(0xffffffffu, a.x, o);
          a.y += __shfl_xor_sync(0xffffffffu, a.y, o);
        }
        if (rl == 0) part[pair * kBMax + q] = a;
      }
      cluster.sync();  // (B) partials of every CTA ready
      if (rank == 0) {
        // sum partials over the cluster in rank order
        for (int e = tid; e < npairs * b; e += kPT) {
          const int pr = e / b, qq = e % b;
          double2 a = make_double2(0.0, 0.0);
          for (int r = 0; r < CS; ++r) a = cadd(a, cluster.map_shared_rank(part, r)[pr * kBMax + qq]);
          tot[pr * kBMax + qq] = a;
        }
        __syncthreads();
        // G' = G - C^H C
        for (int e = tid; e < b * b; e += kPT) {
          const int pp = e / b, qq = e % b;
          double2 g = tot[(nb * b + pp) * kBMax + qq];
          for (int r = 0; r < nb * b; ++r) g = csub(g, cdotc(tot[r * kBMax + pp], tot[r * kBMax + qq]));
          sG[pp * kBMax + qq] = g;
        }
        __syncthreads();
        double2* Rx = (pass == 1) ? R1 : R2;
        double2* Cx = (pass == 1) ? C1 : C2;
        if (tid == 0) {
          double gmax = 0.0;
          for (int pp = 0; pp < b; ++pp) gmax = fmax(gmax, tot[(nb * b + pp) * kBMax + pp].x);
          for (int i = 0; i < kBMax * kBMax; ++i) Rx[i] = make_double2(0.0, 0.0);
          bool ok = gmax > 0.0;
          for (int j = 0; j < b && ok; ++j) {
            double sdg = sG[j * kBMax + j].x;
            for (int k = 0; k < j; ++k) sdg -= Rx[k * kBMax + j].x * Rx[k * kBMax + j].x + Rx[k * kBMax + j].y * Rx[k * kBMax + j].y;
            if (!(sdg > 1e-26 * gmax)) {
              ok = false;
              break;
            }
            const double rjj = sqrt(sdg);
            Rx[j * kBMax + j] = make_double2(rjj, 0.0);
            for (int qq = j + 1; qq < b; ++qq) {
              double2 tt = sG[j * kBMax + qq];
              for (int k = 0; k < j; ++k) tt = csub(tt, cdotc(Rx[k * kBMax + j], Rx[k * kBMax + qq]));
              Rx[j * kBMax + qq] = make_double2(tt.x / rjj, tt.y / rjj);
            }
          }
          ctl[C_OK] = ok;
          if (!ok) {
            ctl[C_STATUS] = RSED_EBREAKDOWN;
            ctl[C_ACTIVE] = 0;
            ctl[C_RESTART] = 0;
          }
        }
        for (int e = tid; e < nb * b * kBMax; e += kPT) Cx[e] = tot[e];
        __syncthreads();
        if (pass == 2 && ctl[C_OK]) {
          // projected matrix: column block cb = nb-1 gets C1 + C2 R1, row block nb gets R2 R1
          const int cb = nb - 1;
          if (nb >= 1) {
            for (int e = tid; e < nb * b * b; e += kPT) {
              const int r = e / b, qq = e % b;
              double2 v = C1[r * kBMax + qq];
              for (int k = 0; k < b; ++k) v = cadd(v, cmul(C2[r * kBMax + k], R1[k * kBMax + qq]));
              P[(int64_t)r * d.pm + cb * b + qq] = v;
            }
            for (int e = tid; e < b * b; e += kPT) {
              const int pp = e / b, qq = e % b;
              double2 v = make_double2(0.0, 0.0);
              for (int k = 0; k < b; ++k) v = cadd(v, cmul(R2[pp * kBMax + k], R1[k * kBMax + qq]));
              P[(int64_t)(nb * b + pp) * d.pm + cb * b + qq] = v;
            }
          }
          __syncthreads();
          const int nbn = nb + 1;
          const bool full = nbn >= d.n_slots + 1;
          if (tid == 0) {
            ctl[C_NB] = nbn;
            ctl[C_NBOLD] = nb;
            ctl[C_ITERS] += 1;
            ctl[C_RESTART] = 0;
          }
          if (full) {
            // projected eigenproblem (blocks 0..nb-1), restart bookkeeping
            const int M = nb * b;
            const int Kp = min(M, max(nev, K));
            double2* A = reinterpret_cast<double2*>(smem + pl.eigA);
            double2* Sv = reinterpret_cast<double2*>(smem + pl.eigS);
            double* Zs = reinterpret_cast<double*>(smem + pl.eigZ);
            for (int i = tid; i < M * M; i += kPT) {
              const int r = i / M, c = i % M;
              const double2 a = P[(int64_t)r * d.pm + c], bt = P[(int64_t)c * d.pm + r];
              A[r * (M + 1) + c] = make_double2(0.5 * (a.x + bt.x), 0.5 * (a.y - bt.y));
            }
            __syncthreads();
            herm_lowest(A, M, Kp, theta, Sv, Zs, tau, dd, ee, red, vv, pw, nullptr);
            double* rv = st.ritz_val + (int64_t)inst * d.pm;
            double2* rvec = reinterpret_cast<double2*>(st.ritz_vec) + (int64_t)inst * d.pm * d.pm;
            double* res = st.resid + (int64_t)inst * d.pm;
            for (int i = tid; i < M * Kp; i += kPT) {
              const int r = i / Kp, j = i % Kp;
              rvec[(int64_t)r * d.pm + j] = Sv[r * Kp + j];
            }
            for (int j = tid; j < Kp; j += kPT) {
              rv[j] = theta[j];
              double a2 = 0.0;
              for (int qq = 0; qq < b; ++qq) {
                double2 v = make_double2(0.0, 0.0);
                for (int pp = 0; pp < b; ++pp)
                  v = cadd(v, cmul(P[(int64_t)(nb * b + qq) * d.pm + (nb - 1) * b + pp], Sv[((nb - 1) * b + pp) * Kp + j]));
                a2 += v.x * v.x + v.y * v.y;
              }
              resj[j] = sqrt(a2);
              res[j] = resj[j];
            }
            __syncthreads();
            if (tid == 0) {
              int nconv = 0;
              for (int j = 0; j < nev; ++j) {
                if (resj[j] <= st.tol * fmax(1.0, fabs(theta[j]))) ++nconv;
                else break;
              }
              ctl[C_NCONV] = nconv;
              if (nconv >= nev) {
                ctl[C_STATUS] = 1;
                ctl[C_ACTIVE] = 0;
              } else if (++ctl[C_RESTARTS] > st.max_restarts) {
                ctl[C_STATUS] = RSED_ENOTCONV;
                ctl[C_ACTIVE] = 0;
              } else {
                ctl[C_RESTART] = 1;
              }
            }
            __syncthreads();
            if (ctl[C_RESTART]) {
              // coupling rows (from the old P) then the new P: diag(theta) + coupling
              for (int i = tid; i < b * K; i += kPT) {
                const int qq = i / K, j = i % K;
                double2 v = make_double2(0.0, 0.0);
                for (int pp = 0; pp < b; ++pp)
                  v = cadd(v, cmul(P[(int64_t)(nb * b + qq) * d.pm + (nb - 1) * b + pp], Sv[((nb - 1) * b + pp) * Kp + j]));
                A[i] = v;  // staged in A (free now)
              }
              __syncthreads();
              for (int i = tid; i < (nbn * b) * (nbn * b); i += kPT) {
                const int r = i / (nbn * b), c = i % (nbn * b);
                P[(int64_t)r * d.pm + c] = make_double2(0.0, 0.0);
              }
              __syncthreads();
              for (int j = tid; j < K; j += kPT) P[(int64_t)j * d.pm + j] = make_double2(theta[j], 0.0);
              for (int i = tid; i < b * K; i += kPT) {
                const int qq = i / K, j = i % K;
                P[(int64_t)(K + qq) * d.pm + j] = A[i];
              }
              for (int i = tid; i < M * K; i += kPT) {
                const int r = i / K, j = i % K;
                Sloc[r * kKeepMax + j] = Sv[r * Kp + j];
              }
              if (tid == 0) ctl[C_NB] = keep + 1;
            }
          }
        }
        __syncthreads();
      }
      cluster.sync();  // (C) C, R (and restart data) ready in CTA 0
      if (!cluster.map_shared_rank(ctl, 0)[C_OK]) break;
      // copy this pass's coefficients from CTA 0
      {
        const double2* Cs = cluster.map_shared_rank(pass == 1 ? C1 : C2, 0);
        const double2* Rs = cluster.map_shared_rank(pass == 1 ? R1 : R2, 0);
        if (rank != 0) {
          double2* Cd = (pass == 1) ? C1 : C2;
          double2* Rd = (pass == 1) ? R1 : R2;
          for (int e = tid; e < nb * b * kBMax; e += kPT) Cd[e] = Cs[e];
          for (int e = tid; e < kBMax * kBMax; e += kPT) Rd[e] = Rs[e];
        }
        __syncthreads();
      }
      // ---- update own rows: W <- (W - V C) R^-1 (pass 1) or new block (pass 2) ----
      {
        const double2* Cx = (pass == 1) ? C1 : C2;
        const double2* Rx = (pass == 1) ? R1 : R2;
        const int rows_per_iter = kPT / b;
        const int qq = tid % b;
        for (int64_t r0 = rb; r0 < re; r0 += rows_per_iter) {
          const int64_t row = r0 + tid / b;
          double2 w = make_double2(0.0, 0.0);
          if (row < re) {
            w = W[row * d.ld + c0 + qq];
            for (int sl = 0; sl < nb; sl += 4) {
              double2 vr[4][kPB];
#pragma unroll
              for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int pp = 0; pp < kPB; ++pp)
                  vr[u][pp] = (sl + u < nb && pp < b) ? V[(int64_t)(sl + u) * slot + row * d.ld + c0 + pp]
                                                     : make_double2(0.0, 0.0);
#pragma unroll
              for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int pp = 0; pp < kPB; ++pp)
                  if (sl + u < nb && pp < b) w = csub(w, cmul(vr[u][pp], Cx[((sl + u) * b + pp) * kBMax + qq]));
            }
          }
          // triangular solve across the b lanes of this row (lanes base..base+b-1)
          const int base = lane - (lane % b);
          double2 acc = make_double2(0.0, 0.0), xq = make_double2(0.0, 0.0);
          for (int pp = 0; pp < b; ++pp) {
            if (qq == pp) {
              const double rr = Rx[pp * kBMax + pp].x;
              xq = make_double2((w.x - acc.x) / rr, (w.y - acc.y) / rr);
            }
            const double xpx = __shfl_sync(0xffffffffu, xq.x, base + pp);
            const double xpy = __shfl_sync(0xffffffffu, xq.y, base + pp);
            if (qq > pp) acc = cadd(acc, cmul(make_double2(xpx, xpy), Rx[pp * kBMax + qq]));
          }
          if (row < re) {
            if (pass == 1) {
              W[row * d.ld + c0 + qq] = xq;
            } else {
              V[(int64_t)nb * slot + row * d.ld + c0 + qq] = xq;
              X[row * d.ld + c0 + qq] = xq;
              if (st.Xf) reinterpret_cast<float2*>(st.Xf)[row * d.ld + c0 + qq] = make_float2((float)xq.x, (float)xq.y);
            }
          }
        }
        __syncthreads();
      }
    }
    // ---- thick restart of own rows ----
    if (cluster.map_shared_rank(ctl, 0)[C_RESTART]) {
      const int nb_old = cluster.map_shared_rank(ctl, 0)[C_NBOLD];  // blocks 0..nb_old-1 + residual nb_old
      const int M = nb_old * b;
      if (rank != 0) {
        const double2* Ss = cluster.map_shared_rank(Sloc, 0);
        for (int e = tid; e < M * kKeepMax; e += kPT) Sloc[e] = Ss[e];
      }
      __syncthreads();
      const int rows_per_iter = kPT / b;
      const int pp = tid % b;
      for (int64_t r0 = rb; r0 < re; r0 += rows_per_iter) {
        const int64_t row = r0 + tid / b;
        double2 acc[kKeepMax];
        for (int t = 0; t < kKeepMax; ++t) acc[t] = make_double2(0.0, 0.0);
        if (row < re) {
          for (int l0 = 0; l0 < M; l0 += 8) {
            double2 v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u)
              v[u] = (l0 + u < M) ? V[(int64_t)((l0 + u) / b) * slot + row * d.ld + c0 + ((l0 + u) % b)]
                                  : make_double2(0.0, 0.0);
#pragma unroll
            for (int u = 0; u < 8; ++u)
              if (l0 + u < M)
                for (int t = 0; t < keep; ++t)
                  acc[t] = cadd(acc[t], cmul(v[u], Sloc[(l0 + u) * kKeepMax + t * b + pp]));
          }
        }
        __syncthreads();  // every read of the old slots of these rows is done
        if (row < re) {
          for (int t = 0; t < keep; ++t) V[(int64_t)t * slot + row * d.ld + c0 + pp] = acc[t];
          V[(int64_t)keep * slot + row * d.ld + c0 + pp] = V[(int64_t)nb_old * slot + row * d.ld + c0 + pp];
        }
        __syncthreads();
      }
    }
  }
  cluster.sync();  // no CTA leaves while another may still read its shared memory
  if (rank == 0 && tid == 0) {
    stt[S_NB] = ctl[C_NB];
    stt[S_ACTIVE] = ctl[C_ACTIVE];
    stt[S_ITERS] = ctl[C_ITERS];
    stt[S_RESTARTS] = ctl[C_RESTARTS];
    stt[S_STATUS] = ctl[C_ACTIVE] ? 0 : ctl[C_STATUS];
    stt[S_NCONV] = ctl[C_NCONV];
    stt[S_RESTART_NB] = 0;
  }
}

PersistLayout persist_layout(size_t base) {
  PersistLayout l{};
  size_t off = align_up(base, 16);
  const size_t g = sizeof(double2) * kPRows * kBMax;
  l.part = off; off += g;
  l.tot = off; off += g;
  l.c1 = off; off += g;
  l.c2 = off; off += g;
  l.r1 = off; off += sizeof(double2) * kBMax * kBMax;
  l.r2 = off; off += sizeof(double2) * kBMax * kBMax;
  l.sg = off; off += sizeof(double2) * kBMax * kBMax;
  l.sloc = off; off += sizeof(double2) * kJacobiMax * kKeepMax;
  l.eigA = off; off += sizeof(double2) * kJacobiMax * (kJacobiMax + 1);
  l.eigS = off; off += sizeof(double2) * kJacobiMax * kKeepMax;
  l.eigZ = off; off += sizeof(double) * kJacobiMax * kKeepMax;
  l.total = align_up(off, 16);
  return l;
}

LzDims make_dims(const rsed_model_t* md, const rsed_sectors_t* sc, const rsed_lanczos_t* st) {
  LzDims d;
  d.n_orb = md->n_orbits;
  d.ld = sc->ld;
  d.n_inst = st->n_inst;
  d.n_slots = st->n_slots;
  d.pm = st->pm;
  d.chunk_rows = st->chunk_rows;
  d.n_chunks = (int)((d.n_orb + d.chunk_rows - 1) / d.chunk_rows);
  d.pslots = st->n_slots + 3;
  return d;
}

int check_lz(const rsed_model_t* md, const rsed_sectors_t* sc, const rsed_lanczos_t* st) {
  RSED_REQUIRE(md && sc && st, RSED_EINVAL, "NULL descriptor");
  RSED_REQUIRE(st->n_inst >= 1 && st->n_slots >= 2, RSED_EINVAL, "bad batch shape");
  RSED_REQUIRE(st->bmax >= 1 && st->bmax <= kBMax, RSED_ERANGE, "block size > %d", kBMax);
  RSED_REQUIRE(st->keep_blocks >= 1 && st->keep_blocks < st->n_slots, RSED_EINVAL, "bad keep_blocks");
  RSED_REQUIRE(st->keep_blocks * st->bmax <= kKeepMax, RSED_ERANGE, "keep*b > %d", kKeepMax);
  RSED_REQUIRE(st->n_slots * st->bmax <= kJacobiMax, RSED_ERANGE, "n_slots*b > %d", kJacobiMax);
  RSED_REQUIRE(st->pm >= (st->n_slots + 1) * st->bmax, RSED_EINVAL, "pm too small");
  RSED_REQUIRE(st->nev >= 1 && st->nev <= st->keep_blocks * 1 * st->bmax, RSED_EINVAL, "bad nev");
  RSED_REQUIRE(st->chunk_rows >= 1, RSED_EINVAL, "bad chunk_rows");
  RSED_REQUIRE(st->V && st->W && st->P && st->coef && st->partial && st->ritz_val && st->ritz_vec &&
                   st->resid && st->state && st->inst_b && st->inst_col0,
               RSED_EINVAL, "Lanczos buffers missing");
  RSED_REQUIRE(st->precision == 64 || (st->precision == 32 && st->Xf), RSED_EINVAL,
               "precision 32 needs the complex64 block buffer");
  const LzDims d = make_dims(md, sc, st);
  const int64_t need = rsed_lanczos_partial_len(d.n_orb, d.chunk_rows, d.n_inst, d.n_slots);
  RSED_REQUIRE(st->partial_len >= need, RSED_ESCRATCH, "partial buffer too small (%lld < %lld)",
               (long long)st->partial_len, (long long)need);
  return RSED_OK;
}

constexpr int kRestartRG = 2;  // row groups per thread iteration of k_lz_restart_rows (keep <= 8)

template <int KM, int RG, int BB>
int launch_restart_rows(const rsed_lanczos_t& st, const LzDims& d, int64_t grid, size_t smem, cudaStream_t stream) {
  static bool attr_set = false;
  if (!attr_set) {
    RSED_TRY_CUDA(cudaFuncSetAttribute(k_lz_restart_rows<KM, RG, BB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       220 * 1024));
    attr_set = true;
  }
  k_lz_restart_rows<KM, RG, BB><<<(unsigned)grid, 256, smem, stream>>>(st, d);
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}

// Thick restart of every instance whose Ritz step asked for one: the
// whole-row form when its coefficients fit shared memory (two blocks per SM
// up to 115 KB, one up to 220 KB), else the per-instance form.
int launch_restart(const rsed_lanczos_t& st, const LzDims& d, cudaStream_t stream) {
  const size_t smem = sizeof(double2) * (size_t)st.n_slots * st.bmax * st.keep_blocks * d.ld +
                      sizeof(int) * (size_t)d.ld;
  if (!(st.reserved & kFlagNoRowRestart) && d.ld <= 256 && smem <= 220 * 1024 && st.keep_blocks <= 16) {
    int dev = 0, n_sm = 148;
    RSED_TRY_CUDA(cudaGetDevice(&dev));
    RSED_TRY_CUDA(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
    const int rows_pg = 256 / d.ld;
    const int rg = st.keep_blocks <= 8 ? kRestartRG : 2;
    const int64_t iters = ((d.n_orb + rows_pg - 1) / rows_pg + rg - 1) / rg;
    const int64_t per_sm = smem <= 115 * 1024 ? 2 : 1;  // 228 KB per SM, 1 KB reserved per block
    const int64_t grid = iters < n_sm * per_sm ? iters : n_sm * per_sm;
    int rc;
    if (st.keep_blocks <= 8) {
      rc = st.bmax <= 1   ? launch_restart_rows<8, kRestartRG, 1>(st, d, grid, smem, stream)
           : st.bmax <= 2 ? launch_restart_rows<8, kRestartRG, 2>(st, d, grid, smem, stream)
           : st.bmax <= 4 ? launch_restart_rows<8, kRestartRG, 4>(st, d, grid, smem, stream)
                          : launch_restart_rows<8, kRestartRG, 8>(st, d, grid, smem, stream);
    } else {
      rc = launch_restart_rows<16, 2, 1>(st, d, grid, smem, stream);  // keep > 8 needs blocks of 1
    }
    if (rc != RSED_OK) return rc;
  } else {
    k_lz_restart<<<(unsigned)(((d.n_orb + 255) / 256) * d.n_inst), 256, 0, stream>>>(st, d);
  }
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}

constexpr int kUpdRG = 4;  // row groups per thread iteration of k_lz_update_rows

template <int BB>
int launch_update_rows(const rsed_lanczos_t& st, const LzDims& d, int pass, size_t smem, int crows,
                       cudaStream_t stream) {
  static bool attr_set = false;
  if (!attr_set) {
    RSED_TRY_CUDA(cudaFuncSetAttribute(k_lz_update_rows<kUpdRG, BB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       160 * 1024));
    attr_set = true;
  }
  const int rows_pg = 256 / d.ld;
  const int64_t groups = (d.n_orb + rows_pg - 1) / rows_pg;
  int dev = 0, n_sm = 148;
  RSED_TRY_CUDA(cudaGetDevice(&dev));
  RSED_TRY_CUDA(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
  const int64_t iters = (groups + kUpdRG - 1) / kUpdRG;  // each block iteration takes kUpdRG row groups
  const int64_t grid = iters < (int64_t)n_sm * 8 ? iters : (int64_t)n_sm * 8;
  k_lz_update_rows<kUpdRG, BB><<<(unsigned)grid, 256, smem, stream>>>(st, d, pass, crows);
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}

int launch_update(const rsed_lanczos_t& st, const LzDims& d, int pass, cudaStream_t stream) {
  // all instances per block when their coefficients fit in shared memory
  const int crows = st.n_slots * st.bmax;
  const size_t smem = sizeof(double2) * ((size_t)crows * d.ld + (size_t)d.n_inst * st.bmax * st.bmax +
                                         kUpdRG * 256) +
                      sizeof(int) * (size_t)d.ld;
  // (three blocks of 256 per SM; above ~64 KB the lower occupancy costs more
  // than whole-row reads save)
  if (d.n_inst >= 2 && d.ld <= 256 && smem <= 64 * 1024) {
    if (st.bmax <= 1) return launch_update_rows<1>(st, d, pass, smem, crows, stream);
    if (st.bmax <= 2) return launch_update_rows<2>(st, d, pass, smem, crows, stream);
    if (st.bmax <= 4) return launch_update_rows<4>(st, d, pass, smem, crows, stream);
    return launch_update_rows<8>(st, d, pass, smem, crows, stream);
  }
  // rows per block: 8 warps x (32 / b) rows; sized for the largest block of the batch
  const int64_t rows_per_block = 8 * (32 / st.bmax);
  k_lz_update<<<(unsigned)(((d.n_orb + rows_per_block - 1) / rows_per_block) * d.n_inst), 256, 0, stream>>>(
      st, d, pass);
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}

// Streaming configuration of a batch: panel rows pr (kPanelElems / ld), ring
// depth ns (the deepest ring, 4..12 stages, that leaves two blocks per SM),
// grid.  False when the batch does not fit the streaming kernels.
struct StreamConfig {
  int pr, ns_gram, ns_upd, grid;
  size_t smem_gram, smem_upd;
};

bool stream_config(const rsed_lanczos_t& st, const LzDims& d, StreamConfig* c) {
  if (st.reserved & kFlagNoStream) return false;
  // lane = column in the Gram loop: below 16 columns most lanes would idle
  // (one sector of block 1 or 2: the per-instance kernel is faster)
  // and below ~32k rows the ring's fill latency outweighs the streaming (a
  // 892-row batch: 12.8 vs 8 ms per step), so small bases keep it too
  if (d.ld < 16 || d.ld > 64 || d.n_inst > kStreamInstMax || d.n_orb < 32768) return false;
  const int crows = st.n_slots * st.bmax;
  constexpr size_t kBudget = 104 * 1024;  // dynamic shared memory per block (two blocks per SM)
  c->pr = kPanelElems / d.ld;
  c->ns_gram = c->ns_upd = 0;
  for (int ns = 12; ns >= 4 && !c->ns_gram; --ns)
    if (stream_layout(ns, d.n_inst, crows, d.ld, false).total <= kBudget) c->ns_gram = ns;
  for (int ns = 12; ns >= 4 && !c->ns_upd; --ns)
    if (stream_layout(ns, d.n_inst, crows, d.ld, true).total <= kBudget) c->ns_upd = ns;
  if (!c->ns_gram || !c->ns_upd) return false;
  c->smem_gram = stream_layout(c->ns_gram, d.n_inst, crows, d.ld, false).total;
  c->smem_upd = stream_layout(c->ns_upd, d.n_inst, crows, d.ld, true).total;
  int dev = 0, n_sm = 148;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return false;
  const int64_t n_rchunks = (d.n_orb + c->pr - 1) / c->pr;
  int64_t grid = 2 * (int64_t)n_sm;
  if (grid > kStreamGridMax) grid = kStreamGridMax;
  if (grid > n_rchunks) grid = n_rchunks;
  c->grid = (int)grid;
  return true;
}

template <int BB, int CPL>
int launch_gram_stream(const rsed_lanczos_t& st, const LzDims& d, int pass, const StreamConfig& c,
                       cudaStream_t stream) {
  static bool attr_set = false;
  if (!attr_set) {
    RSED_TRY_CUDA(cudaFuncSetAttribute(k_lz_gram_stream<BB, CPL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       110 * 1024));
    attr_set = true;
  }
  k_lz_gram_stream<BB, CPL><<<(unsigned)c.grid, kSThreads, c.smem_gram, stream>>>(
      st, d, pass, c.ns_gram, c.pr, st.n_slots * st.bmax);
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}

int launch_pass_stream(const rsed_lanczos_t& st, const LzDims& d, int pass, const StreamConfig& c,
                       cudaStream_t stream) {
  LzDims ds = d;
  ds.n_chunks = c.grid;  // one Gram partial per streaming block
  const int bb = st.bmax <= 1 ? 1 : st.bmax <= 2 ? 2 : st.bmax <= 4 ? 4 : 8;
  int rc;
  if (d.ld <= 32) {
    rc = bb == 1   ? launch_gram_stream<1, 1>(st, ds, pass, c, stream)
         : bb == 2 ? launch_gram_stream<2, 1>(st, ds, pass, c, stream)
         : bb == 4 ? launch_gram_stream<4, 1>(st, ds, pass, c, stream)
                   : launch_gram_stream<8, 1>(st, ds, pass, c, stream);
  } else {
    rc = bb == 1   ? launch_gram_stream<1, 2>(st, ds, pass, c, stream)
         : bb == 2 ? launch_gram_stream<2, 2>(st, ds, pass, c, stream)
         : bb == 4 ? launch_gram_stream<4, 2>(st, ds, pass, c, stream)
                   : launch_gram_stream<8, 2>(st, ds, pass, c, stream);
  }
  if (rc != RSED_OK) return rc;
  k_lz_finalize<<<(unsigned)d.n_inst, kRT, 0, stream>>>(st, ds, pass);
  RSED_CHECK_LAUNCH();
  if (st.reserved & kFlagNoStreamUpdate) return launch_update(st, d, pass, stream);
  static bool attr_set = false;
  if (!attr_set) {
    RSED_TRY_CUDA(cudaFuncSetAttribute(k_lz_update_stream, cudaFuncAttributeMaxDynamicSharedMemorySize, 110 * 1024));
    attr_set = true;
  }
  k_lz_update_stream<<<(unsigned)c.grid, kSThreads, c.smem_upd, stream>>>(st, ds, pass, c.ns_upd, c.pr,
                                                                            st.n_slots * st.bmax);
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}

int launch_pass(const rsed_lanczos_t& st, const LzDims& d, int pass, cudaStream_t stream) {
  StreamConfig sc;
  if (stream_config(st, d, &sc)) return launch_pass_stream(st, d, pass, sc, stream);
  k_lz_reduce<<<(unsigned)(d.n_chunks * d.n_inst), kRT, 0, stream>>>(st, d, pass);
  RSED_CHECK_LAUNCH();
  return launch_update(st, d, pass, stream);
}

__global__ void k_lz_init_state(rsed_lanczos_t st) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= st.n_inst) return;
  int* s = st.state + i * kStateInts;
  s[S_NB] = 0;
  s[S_STATUS] = 0;
  s[S_RESTARTS] = 0;
  s[S_ITERS] = 0;
  s[S_ACTIVE] = 1;
  s[S_RESTART_NB] = 0;
  s[S_NEWSLOT] = 0;
  s[S_NCONV] = 0;
  for (int k = S_TICKET; k < kStateInts; ++k) s[k] = 0;
}

__global__ void k_gather_rows(int64_t n_rows, const int32_t* orbit_of_row, const double2* src,
                              int64_t src_ld, int src_col, double2* dst, int64_t dst_stride) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r < n_rows) dst[r * dst_stride] = src[(int64_t)orbit_of_row[r] * src_ld + src_col];
}

__global__ void k_scatter_rows(int64_t n_rows, const int32_t* orbit_of_row, const double2* src,
                               int64_t src_stride, double2* dst, int64_t dst_ld, int dst_col) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r < n_rows) dst[(int64_t)orbit_of_row[r] * dst_ld + dst_col] = src[r * src_stride];
}

// One thread per (row, column) of a row-major [n_rows, dst_ld] block.
__global__ void k_gather_block(int64_t n_rows, const int32_t* orbit_of_row, const double2* src, int n_cols,
                               int64_t src_col_stride, double2* dst, int64_t dst_ld) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_rows * n_cols) return;
  const int64_t r = e / n_cols;
  const int j = (int)(e - r * n_cols);
  dst[r * dst_ld + j] = src[(int64_t)j * src_col_stride + orbit_of_row[r]];
}

// One thread per (row, column) of a row-major [n_rows, src_ld] block.
__global__ void k_scatter_block(int64_t n_rows, const int32_t* orbit_of_row, const double2* src, int n_cols,
                                int64_t src_ld, double2* dst, int64_t dst_ld, int dst_col0) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_rows * n_cols) return;
  const int64_t r = e / n_cols;
  const int j = (int)(e - r * n_cols);
  dst[(int64_t)orbit_of_row[r] * dst_ld + dst_col0 + j] = src[r * src_ld + j];
}

}  // namespace

extern "C" int64_t rsed_lanczos_partial_len(int64_t n_orbits, int32_t chunk_rows, int32_t n_inst,
                                            int32_t n_slots) {
  int64_t n_chunks = (n_orbits + chunk_rows - 1) / chunk_rows;
  if (n_chunks < kStreamGridMax) n_chunks = kStreamGridMax;  // the streaming reduction's partials
  const int64_t lz = (int64_t)(n_slots + 3) * kBMax * kBMax * 2;
  const int64_t rr = (int64_t)kRRMax * kRRMax * 2;
  return n_chunks * n_inst * (lz > rr ? lz : rr);
}

extern "C" int64_t rsed_lanczos_coef_len(int32_t n_inst, int32_t n_slots) {
  return (int64_t)n_inst * 2 * (n_slots + 3) * kBMax * kBMax * 2;
}

extern "C" int rsed_lanczos_max_block(void) { return kBMax; }
extern "C" int rsed_lanczos_max_keep(void) { return kKeepMax; }
extern "C" int rsed_lanczos_max_projected(void) { return kJacobiMax; }

static int set_ritz_smem() {
  static bool done = false;
  if (!done) {
    RSED_TRY_CUDA(cudaFuncSetAttribute(k_lz_ritz, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kRitzSmem));
    done = true;
  }
  return RSED_OK;
}

extern "C" int rsed_lanczos_prepare(void) { return set_ritz_smem(); }

extern "C" int rsed_lanczos_start(const rsed_model_t* md, const rsed_sectors_t* sc, rsed_lanczos_t* st,
                                  void* stream_) {
  int rc = check_lz(md, sc, st);
  if (rc) return rc;
  cudaStream_t stream = as_stream(stream_);
  const LzDims d = make_dims(md, sc, st);
  k_lz_init_state<<<(st->n_inst + 63) / 64, 64, 0, stream>>>(*st);
  RSED_CHECK_LAUNCH();
  RSED_TRY_CUDA(cudaMemsetAsync(st->P, 0, sizeof(double2) * (size_t)st->n_inst * d.pm * d.pm, stream));
  // start block sits in W: two CholQR passes with an empty basis
  rc = launch_pass(*st, d, 1, stream);
  if (rc) return rc;
  // pass 2 with nb = 0 appends slot 0 and sets nb = 1
  return launch_pass(*st, d, 2, stream);
}

// n_iter iterations: H X, Gram passes 1 and 2, then the Ritz check and the
// restart after every iteration (ritz_mode 0), after the last one only (1)
// or never (2).
static int lz_iterate(const rsed_model_t* md, const rsed_sectors_t* sc, rsed_lanczos_t* st, int32_t n_iter,
                      int ritz_mode, int32_t check_every, int32_t apply_variant, void* stream_) {
  int rc = check_lz(md, sc, st);
  if (rc) return rc;
  rc = set_ritz_smem();
  if (rc) return rc;
  RSED_REQUIRE(check_every >= 1, RSED_EINVAL, "check_every must be >= 1");
  RSED_REQUIRE(n_iter >= 0, RSED_EINVAL, "n_iter must be >= 0");
  cudaStream_t stream = as_stream(stream_);
  const LzDims d = make_dims(md, sc, st);
  const double2* X = reinterpret_cast<const double2*>(st->V) + (int64_t)(st->n_slots + 1) * d.n_orb * d.ld;
  for (int it = 0; it < n_iter; ++it) {
    const void* xin = (st->precision == 32) ? (const void*)st->Xf : (const void*)X;
    rc = rsed_apply_h(md, sc, xin, st->W, st->precision, apply_variant, stream_);
    if (rc) return rc;
    rc = launch_pass(*st, d, 1, stream);
    if (rc) return rc;
    rc = launch_pass(*st, d, 2, stream);
    if (rc) return rc;
    if (ritz_mode == 0 || (ritz_mode == 1 && it == n_iter - 1)) {
      k_lz_ritz<<<d.n_inst, kRitzThreads, kRitzSmem, stream>>>(*st, d, check_every, 0, 0);
      RSED_CHECK_LAUNCH();
      rc = launch_restart(*st, d, stream);
      if (rc) return rc;
    }
  }
  return RSED_OK;
}

extern "C" int rsed_lanczos_iterate(const rsed_model_t* md, const rsed_sectors_t* sc, rsed_lanczos_t* st,
                                    int32_t n_iter, int32_t check_every, int32_t apply_variant,
                                    void* stream_) {
  return lz_iterate(md, sc, st, n_iter, 0, check_every, apply_variant, stream_);
}

extern "C" int rsed_lanczos_iterate_span(const rsed_model_t* md, const rsed_sectors_t* sc, rsed_lanczos_t* st,
                                         int32_t n_iter, int32_t ritz_last, int32_t check_every,
                                         int32_t apply_variant, void* stream_) {
  return lz_iterate(md, sc, st, n_iter, ritz_last ? 1 : 2, check_every, apply_variant, stream_);
}

extern "C" int rsed_lanczos_rayleigh_ritz(const rsed_model_t* md, const rsed_sectors_t* sc,
                                          rsed_lanczos_t* st, int32_t apply_variant, void* stream_) {
  int rc = check_lz(md, sc, st);
  if (rc) return rc;
  rc = set_ritz_smem();
  if (rc) return rc;
  RSED_REQUIRE(st->n_slots >= 2 * st->keep_blocks + 1, RSED_EINVAL,
               "Rayleigh-Ritz needs n_slots >= 2*keep_blocks + 1");
  cudaStream_t stream = as_stream(stream_);
  const LzDims d = make_dims(md, sc, st);
  k_rr_prepare<<<(st->n_inst + 63) / 64, 64, 0, stream>>>(*st);
  RSED_CHECK_LAUNCH();
  rc = launch_restart(*st, d, stream);
  if (rc) return rc;
  const int64_t slot = d.n_orb * d.ld;
  double2* V = reinterpret_cast<double2*>(st->V);
  for (int l = 0; l <= st->keep_blocks; ++l) {
    rc = rsed_apply_h(md, sc, V + l * slot, V + (st->keep_blocks + 1 + l) * slot, 64, apply_variant, stream_);
    if (rc) return rc;
  }
  const unsigned g = (unsigned)(d.n_chunks * d.n_inst);
  k_rr_gram<<<g, 256, 0, stream>>>(*st, d);
  RSED_CHECK_LAUNCH();
  k_lz_ritz<<<d.n_inst, kRitzThreads, kRitzSmem, stream>>>(*st, d, 1, 1, 1);
  RSED_CHECK_LAUNCH();
  k_rr_resid<<<g, 128, 0, stream>>>(*st, d);
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}

extern "C" int rsed_lanczos_persistent(const rsed_model_t* md, const rsed_sectors_t* sc, rsed_lanczos_t* st,
                                       int32_t cluster_size, int32_t max_iter, void* stream_) {
  int rc = check_lz(md, sc, st);
  if (rc) return rc;
  RSED_REQUIRE(cluster_size >= 1 && cluster_size <= 8, RSED_ERANGE, "cluster size %d outside [1, 8]",
               cluster_size);
  RSED_REQUIRE(max_iter >= 1, RSED_EINVAL, "max_iter must be >= 1");
  RSED_REQUIRE(md->n_terms >= 0, RSED_EINVAL, "bad model");
  const LzDims d = make_dims(md, sc, st);
  RSED_REQUIRE(d.n_slots * st->bmax <= kJacobiMax, RSED_ERANGE, "n_slots*b > %d", kJacobiMax);
  RSED_REQUIRE(st->bmax <= kPB, RSED_ERANGE, "the persistent form takes blocks of at most %d", kPB);
  rsed_apply::ApplySmemLayout alay = rsed_apply::apply_layout(*md, *sc);
  PersistLayout pl = persist_layout(alay.total);
  RSED_REQUIRE(pl.total <= 220 * 1024, RSED_ERANGE, "persistent kernel needs %zu B of shared memory",
               pl.total);
  cudaStream_t stream = as_stream(stream_);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(st->n_inst * cluster_size), 1, 1);
  cfg.blockDim = dim3(kPT, 1, 1);
  cfg.dynamicSmemBytes = pl.total;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)cluster_size;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (st->precision == 64) {
    RSED_TRY_CUDA(cudaFuncSetAttribute(k_lz_persist<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pl.total));
    RSED_TRY_CUDA(cudaLaunchKernelEx(&cfg, k_lz_persist<64>, *md, *sc, *st, d, alay, pl, (int)max_iter));
  } else {
    RSED_TRY_CUDA(cudaFuncSetAttribute(k_lz_persist<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pl.total));
    RSED_TRY_CUDA(cudaLaunchKernelEx(&cfg, k_lz_persist<32>, *md, *sc, *st, d, alay, pl, (int)max_iter));
  }
  rsed_count_launch();
  return RSED_OK;
}

extern "C" int rsed_lanczos_restart(const rsed_model_t* md, const rsed_sectors_t* sc, rsed_lanczos_t* st,
                                    void* stream_) {
  int rc = check_lz(md, sc, st);
  if (rc) return rc;
  return launch_restart(*st, make_dims(md, sc, st), as_stream(stream_));
}

extern "C" int rsed_lanczos_extract(const rsed_model_t* md, const rsed_sectors_t* sc, rsed_lanczos_t* st,
                                    double* U, int64_t u_stride, void* stream_) {
  int rc = check_lz(md, sc, st);
  if (rc) return rc;
  RSED_REQUIRE(U != nullptr && u_stride >= md->n_orbits, RSED_EINVAL, "bad U buffer");
  cudaStream_t stream = as_stream(stream_);
  const LzDims d = make_dims(md, sc, st);
  k_lz_extract<<<(unsigned)(((d.n_orb + 255) / 256) * d.n_inst), 256, 0, stream>>>(
      *st, d, reinterpret_cast<double2*>(U), u_stride);
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}

extern "C" int rsed_gather_rows(int64_t n_rows, const int32_t* orbit_of_row, const double* src,
                                int64_t src_ld, int32_t src_col, double* dst, int64_t dst_stride,
                                void* stream_) {
  RSED_REQUIRE(n_rows >= 0 && orbit_of_row && src && dst, RSED_EINVAL, "bad gather arguments");
  if (n_rows == 0) return RSED_OK;
  k_gather_rows<<<(unsigned)((n_rows + 255) / 256), 256, 0, as_stream(stream_)>>>(
      n_rows, orbit_of_row, reinterpret_cast<const double2*>(src), src_ld, src_col,
      reinterpret_cast<double2*>(dst), dst_stride);
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}

extern "C" int rsed_scatter_rows(int64_t n_rows, const int32_t* orbit_of_row, const double* src,
                                 int64_t src_stride, double* dst, int64_t dst_ld, int32_t dst_col,
                                 void* stream_) {
  RSED_REQUIRE(n_rows >= 0 && orbit_of_row && src && dst, RSED_EINVAL, "bad scatter arguments");
  if (n_rows == 0) return RSED_OK;
  k_scatter_rows<<<(unsigned)((n_rows + 255) / 256), 256, 0, as_stream(stream_)>>>(
      n_rows, orbit_of_row, reinterpret_cast<const double2*>(src), src_stride,
      reinterpret_cast<double2*>(dst), dst_ld, dst_col);
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}

extern "C" int rsed_gather_block(int64_t n_rows, const int32_t* orbit_of_row, const double* src, int32_t n_cols,
                                 int64_t src_col_stride, double* dst, int64_t dst_ld, void* stream_) {
  RSED_REQUIRE(n_rows >= 0 && n_cols >= 1 && dst_ld >= n_cols && orbit_of_row && src && dst, RSED_EINVAL,
               "bad gather arguments");
  if (n_rows == 0) return RSED_OK;
  const int64_t n = n_rows * n_cols;
  k_gather_block<<<(unsigned)((n + 255) / 256), 256, 0, as_stream(stream_)>>>(
      n_rows, orbit_of_row, reinterpret_cast<const double2*>(src), n_cols, src_col_stride,
      reinterpret_cast<double2*>(dst), dst_ld);
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}

extern "C" int rsed_scatter_block(int64_t n_rows, const int32_t* orbit_of_row, const double* src,
                                  int32_t n_cols, int64_t src_ld, double* dst, int64_t dst_ld,
                                  int32_t dst_col0, void* stream_) {
  RSED_REQUIRE(n_rows >= 0 && n_cols >= 1 && src_ld >= n_cols && orbit_of_row && src && dst, RSED_EINVAL,
               "bad scatter arguments");
  if (n_rows == 0) return RSED_OK;
  const int64_t n = n_rows * n_cols;
  k_scatter_block<<<(unsigned)((n + 255) / 256), 256, 0, as_stream(stream_)>>>(
      n_rows, orbit_of_row, reinterpret_cast<const double2*>(src), n_cols, src_ld,
      reinterpret_cast<double2*>(dst), dst_ld, dst_col0);
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}
