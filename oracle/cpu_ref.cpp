// CPU restatement (C++17 + OpenMP) of the reference's orbit catalog and
// matrix-free sector apply, for bases the numpy oracle cannot hold.
//
// TEST INFRASTRUCTURE -- the checker, never the product.  Used by tests/ (pinned
// against oracle/port.py, itself pinned to the reference engine) and by
// bench.py as a labelled CPU baseline for the 48-site checkerboard, where the
// reference itself cannot run: its rank fallback for more than 42 sites is
// called with n_site = 0 and returns rank 0 for every mask
// (symmetry_resolved_ed.py:665, 896 -> 404-418).  Here the colex rank is the
// binomial sum over set bits (symmetry_resolved_ed.py:122-140) for any N <= 63.
//
// Catalog: the reference's two-pass sweep (symmetry_resolved_ed.py:346-575).
//   pass 1: for every rank r, the mask m = unrank(r) (SRE:377-394) is a
//           representative iff it is the minimum of its |G| images, each image
//           assembled from per-(g, byte, value) tables (SRE:346-374, 519-528);
//           representatives are numbered in rank order (SRE:530-534);
//   pass 2: per representative and group element g ascending: the image, the
//           angle sum (byte partial sums, bytes in order, SRE:537-543),
//           alpha = exp(i * angle) negated for odd fermionic inversion parity
//           (SRE:544-551), rounded to complex64, written at rank(image): rep
//           index, g, alpha -- later g overwrites (SRE:556-560); stabilizer =
//           {g : image == rep} (SRE:563-571).
// Apply (the device kernel's pull form, y = H^dagger x; equal to H x for the
// reference's zero-flux blocks): per sector row r with representative m and
// every bilinear term (i -> j, t) with i occupied and j empty (SRE:656-660),
// m' = m ^ (1 << i) ^ (1 << j), (c, g, alpha) = table[rank(m')], skipped
// unless c is in the sector; element H[c, r] = t * s_JW * alpha * conj(chi_g)
// * sqrt(S_c / S_r) (SRE:676-687); y[r] += conj(H[c, r]) x[c]; plus
// conj(h_diag[r]) x[r], h_diag the density terms with both sites occupied
// (SRE:641-646).
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

using cd = std::complex<double>;

struct Binom {
  int n, k;
  std::vector<int64_t> t;  // (n + 1) x (k + 1)
  Binom(int n_, int k_) : n(n_), k(k_), t((size_t)(n_ + 1) * (k_ + 1), 0) {
    for (int b = 0; b <= n; ++b) {
      t[(size_t)b * (k + 1)] = 1;
      for (int j = 1; j <= std::min(b, k); ++j)
        t[(size_t)b * (k + 1) + j] = (b > 0 ? t[(size_t)(b - 1) * (k + 1) + j - 1] + (j <= b - 1 ? t[(size_t)(b - 1) * (k + 1) + j] : 0) : 0);
    }
  }
  int64_t operator()(int b, int j) const { return (j > k || j < 0 || b < 0) ? 0 : t[(size_t)b * (k + 1) + j]; }
};

inline int64_t rank_of(uint64_t m, const Binom& bt) {
  int64_t r = 0;
  int j = 1;
  while (m) {
    const int b = __builtin_ctzll(m);
    r += bt(b, j);
    ++j;
    m &= m - 1;
  }
  return r;
}

inline uint64_t unrank_of(int64_t r, int n, int k, const Binom& bt) {
  uint64_t m = 0;
  for (int j = k; j >= 1; --j) {
    int b = j - 1;
    while (b + 1 < n && bt(b + 1, j) <= r) ++b;  // largest b with C(b, j) <= r
    m |= 1ull << b;
    r -= bt(b, j);
  }
  return m;
}

struct Group {
  int n, ng, nbytes;
  std::vector<uint64_t> ptab;  // [g][byte][256] image bits
  std::vector<double> atab;    // [g][byte][256] angle partial sums, bits ascending
  std::vector<uint8_t> perm;   // [g][site]
  Group(int n_, int ng_, const uint8_t* perm_, const double* angle) : n(n_), ng(ng_), nbytes((n_ + 7) / 8) {
    perm.assign(perm_, perm_ + (size_t)ng * n);
    ptab.assign((size_t)ng * nbytes * 256, 0);
    atab.assign((size_t)ng * nbytes * 256, 0.0);
    for (int g = 0; g < ng; ++g)
      for (int b = 0; b < nbytes; ++b)
        for (int v = 0; v < 256; ++v) {
          uint64_t out = 0;
          double ang = 0.0;
          for (int i = 0; i < 8; ++i) {
            const int s = 8 * b + i;
            if (s >= n) break;
            if ((v >> i) & 1) {
              out |= 1ull << perm_[(size_t)g * n + s];
              ang += angle ? angle[(size_t)g * n + s] : 0.0;
            }
          }
          ptab[((size_t)g * nbytes + b) * 256 + v] = out;
          atab[((size_t)g * nbytes + b) * 256 + v] = ang;
        }
  }
  inline uint64_t image(int g, uint64_t m) const {
    uint64_t out = 0;
    const uint64_t* p = &ptab[(size_t)g * nbytes * 256];
    for (int b = 0; b < nbytes; ++b) out |= p[b * 256 + ((m >> (8 * b)) & 0xFF)];
    return out;
  }
  inline double angle_sum(int g, uint64_t m) const {
    double a = 0.0;
    const double* p = &atab[(size_t)g * nbytes * 256];
    for (int b = 0; b < nbytes; ++b) a += p[b * 256 + ((m >> (8 * b)) & 0xFF)];
    return a;
  }
  // number of pairs (i < j) of occupied sites whose images are inverted
  inline int inversions(int g, uint64_t m) const {
    const uint8_t* p = &perm[(size_t)g * n];
    int cnt = 0;
    for (uint64_t a = m; a; a &= a - 1) {
      const int i = __builtin_ctzll(a);
      for (uint64_t b = a & (a - 1); b; b &= b - 1) {
        const int j = __builtin_ctzll(b);
        cnt += p[i] > p[j];
      }
    }
    return cnt;
  }
};

inline bool is_rep(uint64_t m, const Group& G) {
  for (int g = 0; g < G.ng; ++g)
    if (G.image(g, m) < m) return false;
  return true;
}

}  // namespace

extern "C" {

// Representatives per block of 2^16 ranks (pass 1); returns the total.
int64_t rsedcpu_count_orbits(int n, int k, int ng, const uint8_t* perm, int64_t* block_counts, int threads) {
  Binom bt(n, k);
  Group G(n, ng, perm, nullptr);
  const int64_t C = bt(n, k);
  const int64_t nblk = (C + 65535) / 65536;
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t blk = 0; blk < nblk; ++blk) {
    const int64_t r0 = blk * 65536, r1 = std::min(C, r0 + 65536);
    uint64_t m = unrank_of(r0, n, k, bt);
    int64_t cnt = 0;
    for (int64_t r = r0; r < r1; ++r) {
      cnt += is_rep(m, G);
      if (r + 1 < r1) {  // Gosper's successor: next mask with k bits in colex order
        const uint64_t c = m & (~m + 1), s = m + c;
        m = (((m ^ s) >> 2) / c) | s;
      }
    }
    block_counts[blk] = cnt;
  }
  int64_t tot = 0;
  for (int64_t b = 0; b < nblk; ++b) tot += block_counts[b];
  return tot;
}

// Pass 2: representatives (rank order), stabilizer bitmasks and the tables
// rep_rank / rep_sym / rep_amp (complex64 as float pairs) over all C ranks.
int rsedcpu_catalog(int n, int k, int ng, const uint8_t* perm, const double* angle, int fermion,
                    const int64_t* block_counts, uint64_t* reprs, uint64_t* stab_mask, int32_t* rep_rank,
                    int32_t* rep_sym, float* rep_amp, int threads) {
  Binom bt(n, k);
  Group G(n, ng, perm, angle);
  const int64_t C = bt(n, k);
  const int64_t nblk = (C + 65535) / 65536;
  std::vector<int64_t> off(nblk + 1, 0);
  for (int64_t b = 0; b < nblk; ++b) off[b + 1] = off[b] + block_counts[b];
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t blk = 0; blk < nblk; ++blk) {
    const int64_t r0 = blk * 65536, r1 = std::min(C, r0 + 65536);
    uint64_t m = unrank_of(r0, n, k, bt);
    int64_t o = off[blk];
    for (int64_t r = r0; r < r1; ++r) {
      if (is_rep(m, G)) reprs[o++] = m;
      if (r + 1 < r1) {
        const uint64_t c = m & (~m + 1), s = m + c;
        m = (((m ^ s) >> 2) / c) | s;
      }
    }
  }
  const int64_t n_orb = off[nblk];
  // scatter: an image belongs to exactly one orbit, so orbits write disjoint
  // entries; within an orbit g ascending keeps the reference's last writer
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t o = 0; o < n_orb; ++o) {
    const uint64_t m = reprs[o];
    uint64_t sm = 0;
    for (int g = 0; g < ng; ++g) {
      const uint64_t img = G.image(g, m);
      cd a = std::exp(cd(0.0, G.angle_sum(g, m)));
      if (fermion && (G.inversions(g, m) & 1)) a *= cd(-1.0, 0.0);  // as the reference: * (-1 + 0j)
      const int64_t idx = rank_of(img, bt);
      rep_rank[idx] = (int32_t)o;
      rep_sym[idx] = g;
      rep_amp[2 * idx] = (float)a.real();
      rep_amp[2 * idx + 1] = (float)a.imag();
      if (img == m) sm |= 1ull << g;
    }
    stab_mask[o] = sm;
  }
  return 0;
}

// Sector membership (SRE:1484-1546): bit s of member[o] is set iff
// |chi_s(h) - alpha_h| <= atol for every h in Stab(o), alpha_h the unrounded
// phase of the fixed point (SRE:563-571); sqrt_stab[o] = sqrt(|Stab(o)|).
int rsedcpu_members(int n, int ng, const uint8_t* perm, const double* angle, int fermion, int64_t n_orb,
                    const uint64_t* reprs, const uint64_t* stab_mask, int n_sec, const double* chi, double atol,
                    uint64_t* member, int threads) {
  Group G(n, ng, perm, angle);
  const cd* CHI = reinterpret_cast<const cd*>(chi);
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t o = 0; o < n_orb; ++o) {
    const uint64_t m = reprs[o];
    uint64_t bits = (n_sec >= 64) ? ~0ull : ((1ull << n_sec) - 1);
    for (uint64_t sm = stab_mask[o]; sm; sm &= sm - 1) {
      const int h = __builtin_ctzll(sm);
      cd a = std::exp(cd(0.0, G.angle_sum(h, m)));
      if (fermion && (G.inversions(h, m) & 1)) a *= cd(-1.0, 0.0);
      for (int s = 0; s < n_sec; ++s)
        if (!(std::abs(CHI[(size_t)s * ng + h] - a) <= atol)) bits &= ~(1ull << s);
    }
    member[o] = bits;
  }
  return 0;
}

// y[r] (compact sector rows) for x given on the same rows; orbit_of_row and
// row_of_orbit (-1 = not in the sector) map between rows and orbits.
// Terms: term_i / term_j 0-based sites, term_t complex128 amplitudes;
// density: dens_i / dens_j 0-based, dens_v complex128.
int rsedcpu_apply(int n, int k, int ng, int fermion, const int32_t* rep_rank, const int32_t* rep_sym,
                  const float* rep_amp, const uint64_t* reprs, const uint64_t* stab_mask, int64_t n_rows,
                  const int32_t* orbit_of_row, const int32_t* row_of_orbit, const double* chi, int n_terms,
                  const int32_t* term_i, const int32_t* term_j, const double* term_t, int n_dens,
                  const int32_t* dens_i, const int32_t* dens_j, const double* dens_v, const double* x, double* y,
                  int threads) {
  Binom bt(n, k);
  const cd* X = reinterpret_cast<const cd*>(x);
  cd* Y = reinterpret_cast<cd*>(y);
  const cd* CHI = reinterpret_cast<const cd*>(chi);
  const cd* T = reinterpret_cast<const cd*>(term_t);
  const cd* DV = reinterpret_cast<const cd*>(dens_v);
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 2048)
  for (int64_t r = 0; r < n_rows; ++r) {
    const int32_t orb = orbit_of_row[r];
    const uint64_t m = reprs[orb];
    const double sr = std::sqrt((double)__builtin_popcountll(stab_mask[orb]));
    cd hd(0.0, 0.0);
    for (int d = 0; d < n_dens; ++d)
      if (((m >> dens_i[d]) & 1) && ((m >> dens_j[d]) & 1)) hd += DV[d];
    cd acc = std::conj(hd) * X[r];
    for (int t = 0; t < n_terms; ++t) {
      const int i = term_i[t], j = term_j[t];
      if (!((m >> i) & 1) || ((m >> j) & 1)) continue;
      const uint64_t mp = m ^ (1ull << i) ^ (1ull << j);
      const int64_t idx = rank_of(mp, bt);
      const int32_t c = rep_rank[idx];
      const int32_t row = row_of_orbit[c];
      if (row < 0) continue;
      double s = 1.0;
      if (fermion) {
        const int lo = std::min(i, j), hi = std::max(i, j);
        const uint64_t between = hi - lo > 1 ? (((1ull << (hi - lo - 1)) - 1) << (lo + 1)) : 0ull;
        if (__builtin_popcountll(m & between) & 1) s = -1.0;
      }
      const cd alpha((double)rep_amp[2 * idx], (double)rep_amp[2 * idx + 1]);
      const double sc = std::sqrt((double)__builtin_popcountll(stab_mask[c]));
      const cd el = T[t] * s * alpha * std::conj(CHI[rep_sym[idx]]) * (sc / sr);
      acc += std::conj(el) * X[row];
    }
    Y[r] = acc;
  }
  (void)ng;
  return 0;
}

}  // extern "C"
