// K1-K5: combinadic enumeration, orbit-stabilizer catalog, flux phase update
// and sector membership.
//
// Layout in HBM (one catalog):
//   table       C(N,k) x 16 B   rsed_entry_t, indexed by combinadic rank
//   repr_masks  n_orb  x 8 B    representative masks, ascending (= rank order)
//   stab_mask   n_orb  x 8 B    bit g set iff g(rep) == rep
//   stab_off    n_orb+1 x 8 B   exclusive offsets into stab_phase
//   stab_phase  sum|Stab| x 16 B complex128 alpha_h(rep), ascending h
#include <cstring>
#include <mutex>
#include "rsed_internal.cuh"

namespace {

constexpr int kFlagThreads = 256;           // threads per block in the flag pass
constexpr int kRanksPerThread = 32;         // one uint32 bitmap word per thread
constexpr int kRanksPerBlock = kFlagThreads * kRanksPerThread;

struct GroupView {
  const int64_t* binom;
  const uint8_t* perm;
  const double* angle;
  const double2* eta;
};

// Stage the group tables into dynamic shared memory.
__device__ GroupView stage_group(const rsed_group_t& g, unsigned char* smem, size_t binom_off,
                                 size_t perm_off, size_t angle_off, size_t eta_off,
                                 bool with_angle, bool with_eta) {
  const int kp1 = g.n_filled + 1;
  const int nb = (g.n_site + 1) * kp1;
  int64_t* sb = reinterpret_cast<int64_t*>(smem + binom_off);
  for (int i = threadIdx.x; i < nb; i += blockDim.x) sb[i] = g.binom[i];
  const int np = g.n_group * g.n_site;
  uint8_t* sp = smem + perm_off;
  for (int i = threadIdx.x; i < np; i += blockDim.x) sp[i] = g.perm[i];
  GroupView v{sb, sp, nullptr, nullptr};
  if (with_angle) {
    double* sa = reinterpret_cast<double*>(smem + angle_off);
    for (int i = threadIdx.x; i < np; i += blockDim.x) sa[i] = g.angle[i];
    v.angle = sa;
  }
  if (with_eta) {
    double2* se = reinterpret_cast<double2*>(smem + eta_off);
    const double2* ge = reinterpret_cast<const double2*>(g.eta);
    for (int i = threadIdx.x; i < np; i += blockDim.x) se[i] = ge[i];
    v.eta = se;
  }
  __syncthreads();
  return v;
}

__device__ __forceinline__ bool is_representative(uint64_t m, const uint8_t* perm, int n_site,
                                                  int n_group) {
  for (int g = 0; g < n_group; ++g) {
    uint64_t img = rsed_permute(m, perm + g * n_site);
    if (img < m) return false;
  }
  return true;
}

// Walks masks in rank order from rank r0: Gosper's successor for one
// species; for two species the B part advances first and wraps into the A part.
struct RankWalker {
  uint64_t m, ca, cbm;
  int64_t rb;
  bool two;
  RsedSpecies sp;
  __device__ void init(int64_t r0, const rsed_group_t& grp, const int64_t* binom, int kp1) {
    two = grp.species_b != 0ull;
    if (!two) {
      m = rsed_unrank(r0, grp.n_site, grp.n_filled, binom, kp1);
      return;
    }
    sp = rsed_species(grp.species_b, grp.n_site, grp.n_filled, grp.n_filled_b, binom, kp1);
    const int64_t ra = r0 / sp.cb;
    rb = r0 % sp.cb;
    ca = rsed_unrank(ra, sp.na, sp.ka, binom, kp1);
    cbm = rsed_unrank(rb, sp.nb, sp.kb, binom, kp1);
    m = rsed_deposit(ca, sp.sa) | rsed_deposit(cbm, sp.sb);
  }
  // call only while a next rank exists
  __device__ void next() {
    if (!two) {
      m = rsed_gosper_next(m);
      return;
    }
    if (rb + 1 < sp.cb) {
      cbm = rsed_gosper_next(cbm);
      ++rb;
    } else {
      cbm = (sp.kb > 0) ? ((1ull << sp.kb) - 1ull) : 0ull;
      rb = 0;
      ca = rsed_gosper_next(ca);
    }
    m = rsed_deposit(ca, sp.sa) | rsed_deposit(cbm, sp.sb);
  }
};

__device__ __forceinline__ int64_t group_cb(const rsed_group_t& grp, const int64_t* binom, int kp1) {
  return grp.species_b ? binom[__popcll(grp.species_b) * kp1 + grp.n_filled_b] : 1;
}

// Pass 1: representative flags as a bitmap, one 32-rank word per thread
// (symmetry_resolved_ed.py:519-528).
__global__ void k_rep_flags(rsed_group_t grp, uint32_t* bitmap, int64_t* block_count,
                            GroupSmemLayout lay) {
  extern __shared__ __align__(16) unsigned char smem[];
  GroupView gv = stage_group(grp, smem, lay.binom_off, lay.perm_off, 0, 0, false, false);
  __shared__ int64_t warp_sums[kFlagThreads / 32];
  const int kp1 = grp.n_filled + 1;
  const int64_t word = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t r0 = word * kRanksPerThread;
  uint32_t bits = 0;
  if (r0 < grp.n_states) {
    RankWalker w;
    w.init(r0, grp, gv.binom, kp1);
    for (int i = 0; i < kRanksPerThread; ++i) {
      const int64_t r = r0 + i;
      if (r >= grp.n_states) break;
      if (is_representative(w.m, gv.perm, grp.n_site, grp.n_group)) bits |= 1u << i;
      if (r + 1 < grp.n_states) w.next();
    }
    bitmap[word] = bits;
  }
  int c = __popc(bits);
  for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int64_t s = 0;
    for (int w = 0; w < kFlagThreads / 32; ++w) s += warp_sums[w];
    block_count[blockIdx.x] = s;
  }
}

// Pass 2a: representative masks in rank order; rep index = exclusive scan of
// the flags (symmetry_resolved_ed.py:531-532).
__global__ void k_rep_list(rsed_group_t grp, const uint32_t* bitmap, const int64_t* block_off,
                           uint64_t* repr_masks, GroupSmemLayout lay) {
  extern __shared__ __align__(16) unsigned char smem[];
  GroupView gv = stage_group(grp, smem, lay.binom_off, lay.perm_off, 0, 0, false, false);
  __shared__ int warp_tot[kFlagThreads / 32];
  const int kp1 = grp.n_filled + 1;
  const int64_t word = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t r0 = word * kRanksPerThread;
  uint32_t bits = (r0 < grp.n_states) ? bitmap[word] : 0u;
  // block-exclusive prefix of popcounts
  int c = __popc(bits);
  int incl = c;
  const int lane = threadIdx.x & 31;
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_tot[threadIdx.x >> 5] = incl;
  __syncthreads();
  int warp_prefix = 0;
  for (int w = 0; w < (int)(threadIdx.x >> 5); ++w) warp_prefix += warp_tot[w];
  int64_t off = block_off[blockIdx.x] + warp_prefix + (incl - c);
  if (bits) {
    RankWalker w;
    w.init(r0, grp, gv.binom, kp1);
    for (int i = 0; i < kRanksPerThread; ++i) {
      if ((bits >> i) & 1u) repr_masks[off++] = w.m;
      const uint32_t rest = (i < kRanksPerThread - 1) ? (bits >> (i + 1)) : 0u;
      if (rest == 0u) break;
      w.next();
    }
  }
}

// Canonicalisation amplitude of U_g on the representative m as the catalog
// computes it: exp(i * angle-sum) with the fermionic flip
// (symmetry_resolved_ed.py:536-551), except at n_filled in {0, n_site} where
// the reference takes the product form (:483-508).
__device__ __forceinline__ double2 catalog_alpha(uint64_t m, int g, const rsed_group_t& grp,
                                                 const GroupView& gv, bool product_form,
                                                 uint64_t* img) {
  const uint8_t* pg = gv.perm + g * grp.n_site;
  if (product_form) return rsed_phase_product(m, pg, gv.eta + g * grp.n_site, grp.fermionic, img);
  *img = rsed_permute(m, pg);
  double ang = rsed_angle_sum(m, gv.angle + g * grp.n_site, grp.n_site);
  double s, c;
  sincos(ang, &s, &c);
  double2 a = make_double2(c, s);
  if (grp.fermionic && rsed_perm_parity(m, pg)) a = rsed_cmul_exact(a, make_double2(-1.0, 0.0));
  return a;
}

// Pass 2b: orbit expansion into the representative table, g ascending so the
// last writer wins for stabilizer cosets (symmetry_resolved_ed.py:553-560),
// plus the stabilizer bitmask (:563).
__global__ void k_expand(rsed_group_t grp, int64_t n_orb, const uint64_t* repr_masks,
                         RsedEntry* table, uint64_t* stab_mask, GroupSmemLayout lay, int* err) {
  extern __shared__ __align__(16) unsigned char smem[];
  const bool product_form = (grp.n_filled == 0 || grp.n_filled == grp.n_site);
  GroupView gv = stage_group(grp, smem, lay.binom_off, lay.perm_off, lay.angle_off, lay.eta_off,
                             true, product_form);
  const int kp1 = grp.n_filled + 1;
  const int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= n_orb) return;
  const uint64_t m = repr_masks[o];
  uint64_t smask = 0;
  for (int g = 0; g < grp.n_group; ++g) {
    uint64_t img;
    double2 a = catalog_alpha(m, g, grp, gv, product_form, &img);
    int64_t idx = rsed_rank_any(img, gv.binom, kp1, grp.species_b, group_cb(grp, gv.binom, kp1));
    if (idx < 0 || idx >= grp.n_states) {
      rsed_flag_error(err, 1);
      continue;
    }
    RsedEntry e;
    e.rep = (int32_t)o;
    e.g = g;
    e.re = __double2float_rn(a.x);
    e.im = __double2float_rn(a.y);
    table[idx] = e;
    if (img == m) smask |= 1ull << g;
  }
  stab_mask[o] = smask;
}

// Entries start as (rep -1, g 0, alpha 0), the reference's initial table
// (symmetry_resolved_ed.py:1359-1361); every state of a group's catalog is
// overwritten by k_expand.
__global__ void k_table_init(int64_t n, RsedEntry* table) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    RsedEntry e;
    e.rep = -1;
    e.g = 0;
    e.re = 0.0f;
    e.im = 0.0f;
    table[i] = e;
  }
}

__global__ void k_stab_counts(int64_t n_orb, const uint64_t* stab_mask, int64_t* counts) {
  int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (o < n_orb) counts[o] = __popcll(stab_mask[o]);
}

// Stabilizer phases (complex128), ascending g (symmetry_resolved_ed.py:563-571).
__global__ void k_stab_phases(rsed_group_t grp, int64_t n_orb, const uint64_t* repr_masks,
                              const uint64_t* stab_mask, const int64_t* stab_off,
                              double2* stab_phase, GroupSmemLayout lay) {
  extern __shared__ __align__(16) unsigned char smem[];
  const bool product_form = (grp.n_filled == 0 || grp.n_filled == grp.n_site);
  GroupView gv = stage_group(grp, smem, lay.binom_off, lay.perm_off, lay.angle_off, lay.eta_off,
                             true, product_form);
  const int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= n_orb) return;
  const uint64_t m = repr_masks[o];
  uint64_t s = stab_mask[o];
  int64_t off = stab_off[o];
  while (s) {
    int g = __ffsll((long long)s) - 1;
    uint64_t img;
    stab_phase[off++] = catalog_alpha(m, g, grp, gv, product_form, &img);
    s &= s - 1;
  }
}

// K4: flux phase update in product form (symmetry_resolved_ed.py:1248-1268).
__global__ void k_phase_update(rsed_group_t grp, int64_t n_orb, const uint64_t* repr_masks,
                               const uint64_t* stab_mask, const int64_t* stab_off,
                               double2* stab_phase, RsedEntry* table, GroupSmemLayout lay,
                               int* err) {
  extern __shared__ __align__(16) unsigned char smem[];
  GroupView gv = stage_group(grp, smem, lay.binom_off, lay.perm_off, 0, lay.eta_off, false, true);
  const int kp1 = grp.n_filled + 1;
  const int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= n_orb) return;
  const uint64_t m = repr_masks[o];
  // stabilizer phases first (reference order: :1248-1257)
  uint64_t s = stab_mask[o];
  int64_t off = stab_off[o];
  while (s) {
    int g = __ffsll((long long)s) - 1;
    uint64_t img;
    stab_phase[off++] =
        rsed_phase_product(m, gv.perm + g * grp.n_site, gv.eta + g * grp.n_site, grp.fermionic, &img);
    s &= s - 1;
  }
  for (int g = 0; g < grp.n_group; ++g) {
    uint64_t img;
    double2 a =
        rsed_phase_product(m, gv.perm + g * grp.n_site, gv.eta + g * grp.n_site, grp.fermionic, &img);
    int64_t idx = rsed_rank_any(img, gv.binom, kp1, grp.species_b, group_cb(grp, gv.binom, kp1));
    if (idx < 0 || idx >= grp.n_states) {
      rsed_flag_error(err, 1);
      continue;
    }
    if (table[idx].rep != (int32_t)o) {
      rsed_flag_error(err, 2);
      continue;
    }
    RsedEntry e;
    e.rep = (int32_t)o;
    e.g = g;
    e.re = __double2float_rn(a.x);
    e.im = __double2float_rn(a.y);
    table[idx] = e;
  }
}

// K5: sector membership for many irreps at once (symmetry_resolved_ed.py:1484-1512).
__global__ void k_sector_members(int64_t n_orb, int n_group, int n_sec, const uint64_t* stab_mask,
                                 const int64_t* stab_off, const double2* stab_phase,
                                 const double2* chi, double atol, uint64_t* member,
                                 double* sqrt_stab, unsigned long long* dims) {
  extern __shared__ __align__(16) unsigned char smem[];
  double2* schi = reinterpret_cast<double2*>(smem);
  for (int i = threadIdx.x; i < n_sec * n_group; i += blockDim.x) schi[i] = chi[i];
  __shared__ unsigned int bcount[64];
  for (int i = threadIdx.x; i < 64; i += blockDim.x) bcount[i] = 0;
  __syncthreads();
  const int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (o < n_orb) {
    const uint64_t sm = stab_mask[o];
    const int64_t off = stab_off[o];
    uint64_t bits = 0;
    for (int s = 0; s < n_sec; ++s) {
      bool ok = true;
      uint64_t t = sm;
      int64_t j = off;
      while (t) {
        int g = __ffsll((long long)t) - 1;
        double2 a = stab_phase[j++];
        double2 c = schi[s * n_group + g];
        if (!(hypot(c.x - a.x, c.y - a.y) <= atol)) {
          ok = false;
          break;
        }
        t &= t - 1;
      }
      if (ok) {
        bits |= 1ull << s;
        atomicAdd(&bcount[s], 1u);
      }
    }
    member[o] = bits;
    sqrt_stab[o] = sqrt((double)__popcll(sm));
  }
  __syncthreads();
  for (int s = threadIdx.x; s < n_sec; s += blockDim.x)
    if (bcount[s]) atomicAdd(&dims[s], (unsigned long long)bcount[s]);
}

__global__ void k_member_bit(int64_t n, const uint64_t* member, int sector, int64_t* out) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (member[i] >> sector) & 1ull;
}

__global__ void k_sector_rows(int64_t n, const uint64_t* member, int sector, const int64_t* pos,
                              int32_t* orbit_of_row, int32_t* row_of_orbit) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if ((member[i] >> sector) & 1ull) {
    int64_t r = pos[i];
    if (orbit_of_row) orbit_of_row[r] = (int32_t)i;
    if (row_of_orbit) row_of_orbit[i] = (int32_t)r;
  } else if (row_of_orbit) {
    row_of_orbit[i] = -1;
  }
}

// Density-density diagonal per orbit in term order (symmetry_resolved_ed.py:641-646).
__global__ void k_density_diag(int64_t n_orb, const uint64_t* repr_masks, int nd, const uint8_t* di,
                               const uint8_t* dj, const double2* dv, double2* hdiag) {
  int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= n_orb) return;
  uint64_t m = repr_masks[o];
  double2 h = make_double2(0.0, 0.0);
  for (int d = 0; d < nd; ++d) {
    if (((m >> di[d]) & 1ull) && ((m >> dj[d]) & 1ull)) {
      h.x = __dadd_rn(h.x, dv[d].x);
      h.y = __dadd_rn(h.y, dv[d].y);
    }
  }
  hdiag[o] = h;
}

// ---- generic exclusive scan -------------------------------------------------
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ int64_t block_exclusive_scan(int64_t v, int64_t* total) {
  __shared__ int64_t ws[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nw = (int)(blockDim.x >> 5);
  int64_t incl = v;
  for (int o = 1; o < 32; o <<= 1) {
    int64_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) ws[w] = incl;
  __syncthreads();
  if (w == 0) {
    int64_t x = (lane < nw) ? ws[lane] : 0;
    int64_t xi = x;
    for (int o = 1; o < 32; o <<= 1) {
      int64_t t = __shfl_up_sync(0xffffffffu, xi, o);
      if (lane >= o) xi += t;
    }
    ws[lane] = xi - x;
    if (lane == nw - 1) *total = xi;
  }
  __syncthreads();
  int64_t r = ws[w] + (incl - v);
  __syncthreads();
  return r;
}

__global__ void k_tile_sums(const int64_t* in, int64_t n, int64_t* tile_sum) {
  __shared__ int64_t tot;
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  int64_t s = 0;
  for (int j = 0; j < kScanItems; ++j) {
    int64_t i = base + (int64_t)threadIdx.x * kScanItems + j;
    if (i < n) s += in[i];
  }
  block_exclusive_scan(s, &tot);
  if (threadIdx.x == 0) tile_sum[blockIdx.x] = tot;
}

__global__ void k_scan_tiles(int64_t* tile_sum, int64_t n_tiles, int64_t* total_out) {
  __shared__ int64_t tot;
  int64_t carry = 0;
  for (int64_t base = 0; base < n_tiles; base += kScanThreads) {
    int64_t i = base + threadIdx.x;
    int64_t v = i < n_tiles ? tile_sum[i] : 0;
    int64_t ex = block_exclusive_scan(v, &tot);
    if (i < n_tiles) tile_sum[i] = carry + ex;
    carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total_out = carry;
}

__global__ void k_tile_scan(const int64_t* in, int64_t n, const int64_t* tile_off,
                            const int64_t* total, int64_t* out) {
  __shared__ int64_t tot;
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int64_t v[kScanItems];
  int64_t s = 0;
  for (int j = 0; j < kScanItems; ++j) {
    int64_t i = base + j;
    v[j] = i < n ? in[i] : 0;
    s += v[j];
  }
  int64_t ex = block_exclusive_scan(s, &tot) + tile_off[blockIdx.x];
  for (int j = 0; j < kScanItems; ++j) {
    int64_t i = base + j;
    if (i < n) out[i] = ex;
    ex += v[j];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = *total;
}

}  // namespace

// ---- host ------------------------------------------------------------------

size_t rsed_scan_scratch_bytes(int64_t n) {
  int64_t tiles = (n + kScanTile - 1) / kScanTile;
  if (tiles < 1) tiles = 1;
  return align_up((size_t)(tiles + 1) * sizeof(int64_t), 256);
}

int rsed_exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t n, void* scratch,
                            size_t scratch_bytes, cudaStream_t stream) {
  int64_t tiles = (n + kScanTile - 1) / kScanTile;
  if (tiles < 1) tiles = 1;
  RSED_REQUIRE(scratch_bytes >= rsed_scan_scratch_bytes(n), RSED_ESCRATCH, "scan scratch too small");
  int64_t* tile_sum = reinterpret_cast<int64_t*>(scratch);
  int64_t* total = tile_sum + tiles;
  if (n == 0) {
    RSED_TRY_CUDA(cudaMemsetAsync(out, 0, sizeof(int64_t), stream));
    return RSED_OK;
  }
  k_tile_sums<<<(unsigned)tiles, kScanThreads, 0, stream>>>(in, n, tile_sum);
  RSED_CHECK_LAUNCH();
  k_scan_tiles<<<1, kScanThreads, 0, stream>>>(tile_sum, tiles, total);
  RSED_CHECK_LAUNCH();
  k_tile_scan<<<(unsigned)tiles, kScanThreads, 0, stream>>>(in, n, tile_sum, total, out);
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}

GroupSmemLayout group_smem_layout(int n_site, int n_filled, int n_group, bool with_eta,
                                  bool with_angle) {
  GroupSmemLayout l{};
  size_t off = 0;
  l.binom_off = off;
  off = align_up(off + sizeof(int64_t) * (size_t)(n_site + 1) * (size_t)(n_filled + 1), 16);
  l.angle_off = off;
  if (with_angle) off = align_up(off + sizeof(double) * (size_t)n_group * n_site, 16);
  l.eta_off = off;
  if (with_eta) off = align_up(off + 2 * sizeof(double) * (size_t)n_group * n_site, 16);
  l.perm_off = off;
  off = align_up(off + (size_t)n_group * n_site, 16);
  l.total = off;
  return l;
}

// Worst-case staged group (63 sites, 31 particles, |G| = 64) needs ~115 KB.
static int set_catalog_smem_limits() {
  static bool done = false;
  if (done) return RSED_OK;
  const int big = 160 * 1024;
  RSED_TRY_CUDA(cudaFuncSetAttribute(k_rep_flags, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  RSED_TRY_CUDA(cudaFuncSetAttribute(k_rep_list, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  RSED_TRY_CUDA(cudaFuncSetAttribute(k_expand, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  RSED_TRY_CUDA(cudaFuncSetAttribute(k_stab_phases, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  RSED_TRY_CUDA(cudaFuncSetAttribute(k_phase_update, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  RSED_TRY_CUDA(cudaFuncSetAttribute(k_sector_members, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  done = true;
  return RSED_OK;
}

int check_group(const rsed_group_t* g) {
  RSED_REQUIRE(g != nullptr, RSED_EINVAL, "group descriptor is NULL");
  RSED_REQUIRE(g->n_site >= 1 && g->n_site <= RSED_MAX_SITES, RSED_ERANGE,
               "n_site = %d outside [1, %d]", g->n_site, RSED_MAX_SITES);
  RSED_REQUIRE(g->n_filled >= 0 && g->n_filled <= g->n_site, RSED_EINVAL,
               "n_filled = %d outside [0, n_site]", g->n_filled);
  RSED_REQUIRE(g->n_group >= 1 && g->n_group <= RSED_MAX_GROUP, RSED_ERANGE,
               "|G| = %d outside [1, %d]", g->n_group, RSED_MAX_GROUP);
  RSED_REQUIRE(g->n_states >= 1, RSED_EINVAL, "n_states must be >= 1");
  RSED_REQUIRE(g->binom && g->perm, RSED_EINVAL, "group tables missing");
  if (g->species_b) {
    const uint64_t all = (g->n_site >= 64) ? ~0ull : ((1ull << g->n_site) - 1ull);
    const int nb = __builtin_popcountll(g->species_b);
    RSED_REQUIRE((g->species_b & ~all) == 0ull && nb < g->n_site, RSED_EINVAL,
                 "species_b must mark a proper subset of the sites");
    RSED_REQUIRE(g->n_filled_b >= 0 && g->n_filled_b <= nb && g->n_filled_b <= g->n_filled &&
                     g->n_filled - g->n_filled_b <= g->n_site - nb,
                 RSED_EINVAL, "n_filled_b = %d does not fit the two species", g->n_filled_b);
  }
  return RSED_OK;
}

namespace {
struct CatalogScratch {
  uint32_t* bitmap;
  int64_t* block_count;
  int64_t* block_off;  // n_blocks + 1
  void* scan;
  size_t scan_bytes;
  int64_t n_blocks, n_words;
};

CatalogScratch carve_catalog_scratch(const rsed_group_t* g, void* base) {
  CatalogScratch s{};
  s.n_words = (g->n_states + kRanksPerThread - 1) / kRanksPerThread;
  s.n_blocks = (g->n_states + kRanksPerBlock - 1) / kRanksPerBlock;
  char* p = reinterpret_cast<char*>(base);
  size_t off = 0;
  s.bitmap = reinterpret_cast<uint32_t*>(p + off);
  off = align_up(off + sizeof(uint32_t) * (size_t)(s.n_blocks * kFlagThreads), 256);
  s.block_count = reinterpret_cast<int64_t*>(p + off);
  off = align_up(off + sizeof(int64_t) * (size_t)s.n_blocks, 256);
  s.block_off = reinterpret_cast<int64_t*>(p + off);
  off = align_up(off + sizeof(int64_t) * (size_t)(s.n_blocks + 1), 256);
  s.scan = p + off;
  s.scan_bytes = rsed_scan_scratch_bytes(s.n_blocks);
  return s;
}
}  // namespace

extern "C" size_t rsed_catalog_scratch_bytes(const rsed_group_t* g) {
  if (!g || g->n_states < 1) return 0;
  int64_t n_blocks = (g->n_states + kRanksPerBlock - 1) / kRanksPerBlock;
  size_t b = align_up(sizeof(uint32_t) * (size_t)(n_blocks * kFlagThreads), 256);
  b += align_up(sizeof(int64_t) * (size_t)n_blocks, 256);
  b += align_up(sizeof(int64_t) * (size_t)(n_blocks + 1), 256);
  b += rsed_scan_scratch_bytes(n_blocks);
  return b;
}

extern "C" int rsed_catalog_count(const rsed_group_t* g, void* scratch, size_t scratch_bytes,
                                  int64_t* n_orbits_out, void* stream_) {
  int rc = check_group(g);
  if (rc) return rc;
  RSED_REQUIRE(scratch_bytes >= rsed_catalog_scratch_bytes(g), RSED_ESCRATCH,
               "catalog scratch too small (%zu < %zu)", scratch_bytes, rsed_catalog_scratch_bytes(g));
  RSED_REQUIRE(n_orbits_out != nullptr, RSED_EINVAL, "n_orbits_out is NULL");
  cudaStream_t stream = as_stream(stream_);
  rc = set_catalog_smem_limits();
  if (rc) return rc;
  CatalogScratch s = carve_catalog_scratch(g, scratch);
  GroupSmemLayout lay = group_smem_layout(g->n_site, g->n_filled, g->n_group, false, false);
  k_rep_flags<<<(unsigned)s.n_blocks, kFlagThreads, lay.total, stream>>>(*g, s.bitmap,
                                                                          s.block_count, lay);
  RSED_CHECK_LAUNCH();
  rc = rsed_exclusive_scan_i64(s.block_count, s.block_off, s.n_blocks, s.scan, s.scan_bytes, stream);
  if (rc) return rc;
  int64_t n_orb = 0;
  RSED_TRY_CUDA(cudaMemcpyAsync(&n_orb, s.block_off + s.n_blocks, sizeof(int64_t),
                                cudaMemcpyDeviceToHost, stream));
  RSED_TRY_CUDA(cudaStreamSynchronize(stream));
  RSED_REQUIRE(n_orb < (int64_t)INT32_MAX, RSED_ERANGE, "more than 2^31-1 orbits");
  *n_orbits_out = n_orb;
  return RSED_OK;
}

extern "C" int rsed_catalog_fill(const rsed_group_t* g, const void* scratch, size_t scratch_bytes,
                                 int64_t n_orbits, uint64_t* repr_masks, rsed_entry_t* table,
                                 uint64_t* stab_mask, void* stream_) {
  int rc = check_group(g);
  if (rc) return rc;
  RSED_REQUIRE(scratch_bytes >= rsed_catalog_scratch_bytes(g), RSED_ESCRATCH,
               "catalog scratch too small");
  RSED_REQUIRE(g->angle != nullptr && g->eta != nullptr, RSED_EINVAL, "group phases missing");
  RSED_REQUIRE(n_orbits >= 1 && repr_masks && table && stab_mask, RSED_EINVAL,
               "catalog outputs missing");
  cudaStream_t stream = as_stream(stream_);
  CatalogScratch s = carve_catalog_scratch(g, const_cast<void*>(scratch));
  GroupSmemLayout lay0 = group_smem_layout(g->n_site, g->n_filled, g->n_group, false, false);
  k_rep_list<<<(unsigned)s.n_blocks, kFlagThreads, lay0.total, stream>>>(*g, s.bitmap, s.block_off,
                                                                          repr_masks, lay0);
  RSED_CHECK_LAUNCH();
  GroupSmemLayout lay = group_smem_layout(g->n_site, g->n_filled, g->n_group, true, true);
  int* err = reinterpret_cast<int*>(s.block_count);  // block counts are consumed by now
  RSED_TRY_CUDA(cudaMemsetAsync(err, 0, sizeof(int), stream));
  k_table_init<<<(unsigned)((g->n_states + 255) / 256), 256, 0, stream>>>(
      g->n_states, reinterpret_cast<RsedEntry*>(table));
  RSED_CHECK_LAUNCH();
  const unsigned nb = (unsigned)((n_orbits + 255) / 256);
  k_expand<<<nb, 256, lay.total, stream>>>(*g, n_orbits, repr_masks,
                                           reinterpret_cast<RsedEntry*>(table), stab_mask, lay, err);
  RSED_CHECK_LAUNCH();
  int herr = 0;
  RSED_TRY_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, stream));
  RSED_TRY_CUDA(cudaStreamSynchronize(stream));
  RSED_REQUIRE(herr == 0, RSED_EINVAL, "catalog expansion produced an out-of-range rank");
  return RSED_OK;
}

extern "C" size_t rsed_stab_scratch_bytes(int64_t n_orbits) {
  return align_up(sizeof(int64_t) * (size_t)(n_orbits + 1), 256) + rsed_scan_scratch_bytes(n_orbits);
}

extern "C" int rsed_catalog_stab_count(int64_t n_orbits, const uint64_t* stab_mask, int64_t* stab_off,
                                       int64_t* n_stab_out, void* scratch, size_t scratch_bytes,
                                       void* stream_) {
  RSED_REQUIRE(n_orbits >= 1 && stab_mask && stab_off && n_stab_out, RSED_EINVAL,
               "bad stabilizer-count arguments");
  RSED_REQUIRE(scratch_bytes >= rsed_stab_scratch_bytes(n_orbits), RSED_ESCRATCH,
               "stabilizer scratch too small");
  cudaStream_t stream = as_stream(stream_);
  int64_t* counts = reinterpret_cast<int64_t*>(scratch);
  char* scan = reinterpret_cast<char*>(scratch) + align_up(sizeof(int64_t) * (size_t)(n_orbits + 1), 256);
  k_stab_counts<<<(unsigned)((n_orbits + 255) / 256), 256, 0, stream>>>(n_orbits, stab_mask, counts);
  RSED_CHECK_LAUNCH();
  int rc = rsed_exclusive_scan_i64(counts, stab_off, n_orbits, scan, rsed_scan_scratch_bytes(n_orbits),
                                   stream);
  if (rc) return rc;
  RSED_TRY_CUDA(cudaMemcpyAsync(n_stab_out, stab_off + n_orbits, sizeof(int64_t),
                                cudaMemcpyDeviceToHost, stream));
  RSED_TRY_CUDA(cudaStreamSynchronize(stream));
  return RSED_OK;
}

extern "C" int rsed_catalog_stab(const rsed_group_t* g, int64_t n_orbits, const uint64_t* repr_masks,
                                 const uint64_t* stab_mask, const int64_t* stab_off,
                                 double* stab_phase, void* stream_) {
  int rc = check_group(g);
  if (rc) return rc;
  RSED_REQUIRE(g->angle != nullptr && g->eta != nullptr, RSED_EINVAL, "group phases missing");
  RSED_REQUIRE(n_orbits >= 1 && repr_masks && stab_mask && stab_off && stab_phase, RSED_EINVAL,
               "bad stabilizer arguments");
  cudaStream_t stream = as_stream(stream_);
  rc = set_catalog_smem_limits();
  if (rc) return rc;
  GroupSmemLayout lay = group_smem_layout(g->n_site, g->n_filled, g->n_group, true, true);
  k_stab_phases<<<(unsigned)((n_orbits + 255) / 256), 256, lay.total, stream>>>(
      *g, n_orbits, repr_masks, stab_mask, stab_off, reinterpret_cast<double2*>(stab_phase), lay);
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}

extern "C" int rsed_phase_update(const rsed_group_t* g, int64_t n_orbits, const uint64_t* repr_masks,
                                 const uint64_t* stab_mask, const int64_t* stab_off,
                                 double* stab_phase, rsed_entry_t* table, int* err_dev,
                                 void* stream_) {
  int rc = check_group(g);
  if (rc) return rc;
  RSED_REQUIRE(g->eta != nullptr, RSED_EINVAL, "group phases missing");
  RSED_REQUIRE(n_orbits >= 1 && repr_masks && stab_mask && stab_off && stab_phase && table && err_dev,
               RSED_EINVAL, "bad phase-update arguments");
  cudaStream_t stream = as_stream(stream_);
  rc = set_catalog_smem_limits();
  if (rc) return rc;
  GroupSmemLayout lay = group_smem_layout(g->n_site, g->n_filled, g->n_group, true, false);
  RSED_TRY_CUDA(cudaMemsetAsync(err_dev, 0, sizeof(int), stream));
  k_phase_update<<<(unsigned)((n_orbits + 255) / 256), 256, lay.total, stream>>>(
      *g, n_orbits, repr_masks, stab_mask, stab_off, reinterpret_cast<double2*>(stab_phase),
      reinterpret_cast<RsedEntry*>(table), lay, err_dev);
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}

extern "C" size_t rsed_sector_scratch_bytes(int64_t n_orbits, int32_t n_sectors) {
  (void)n_sectors;
  return align_up(sizeof(int64_t) * (size_t)(n_orbits + 1), 256) * 2 +
         rsed_scan_scratch_bytes(n_orbits);
}

extern "C" int rsed_sector_members(int64_t n_orbits, int32_t n_group, int32_t n_sectors,
                                   const uint64_t* stab_mask, const int64_t* stab_off,
                                   const double* stab_phase, const double* chi, double atol,
                                   uint64_t* member, double* sqrt_stab, int64_t* sector_dims,
                                   void* stream_) {
  RSED_REQUIRE(n_orbits >= 1 && n_group >= 1 && n_group <= RSED_MAX_GROUP, RSED_EINVAL,
               "bad sector arguments");
  RSED_REQUIRE(n_sectors >= 1 && n_sectors <= 64, RSED_ERANGE, "n_sectors = %d outside [1, 64]",
               n_sectors);
  RSED_REQUIRE(stab_mask && stab_off && stab_phase && chi && member && sqrt_stab && sector_dims,
               RSED_EINVAL, "sector buffers missing");
  cudaStream_t stream = as_stream(stream_);
  int rc = set_catalog_smem_limits();
  if (rc) return rc;
  RSED_TRY_CUDA(cudaMemsetAsync(sector_dims, 0, sizeof(int64_t) * n_sectors, stream));
  size_t smem = sizeof(double2) * (size_t)n_sectors * n_group;
  k_sector_members<<<(unsigned)((n_orbits + 255) / 256), 256, smem, stream>>>(
      n_orbits, n_group, n_sectors, stab_mask, stab_off, reinterpret_cast<const double2*>(stab_phase),
      reinterpret_cast<const double2*>(chi), atol, member, sqrt_stab,
      reinterpret_cast<unsigned long long*>(sector_dims));
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}

extern "C" int rsed_sector_rows(int64_t n_orbits, const uint64_t* member, int32_t sector,
                                int32_t* orbit_of_row, int32_t* row_of_orbit, void* scratch,
                                size_t scratch_bytes, void* stream_) {
  RSED_REQUIRE(n_orbits >= 1 && member && sector >= 0 && sector < 64, RSED_EINVAL,
               "bad sector-rows arguments");
  RSED_REQUIRE(scratch_bytes >= rsed_sector_scratch_bytes(n_orbits, 1), RSED_ESCRATCH,
               "sector scratch too small");
  cudaStream_t stream = as_stream(stream_);
  char* p = reinterpret_cast<char*>(scratch);
  size_t a = align_up(sizeof(int64_t) * (size_t)(n_orbits + 1), 256);
  int64_t* flags = reinterpret_cast<int64_t*>(p);
  int64_t* pos = reinterpret_cast<int64_t*>(p + a);
  const unsigned nb = (unsigned)((n_orbits + 255) / 256);
  k_member_bit<<<nb, 256, 0, stream>>>(n_orbits, member, sector, flags);
  RSED_CHECK_LAUNCH();
  int rc = rsed_exclusive_scan_i64(flags, pos, n_orbits, p + 2 * a, rsed_scan_scratch_bytes(n_orbits),
                                   stream);
  if (rc) return rc;
  k_sector_rows<<<nb, 256, 0, stream>>>(n_orbits, member, sector, pos, orbit_of_row, row_of_orbit);
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}

extern "C" int rsed_density_diag(int64_t n_orbits, const uint64_t* repr_masks, int32_t n_density,
                                 const uint8_t* dens_i, const uint8_t* dens_j, const double* dens_v,
                                 double* hdiag, void* stream_) {
  RSED_REQUIRE(n_orbits >= 1 && repr_masks && hdiag && n_density >= 0, RSED_EINVAL,
               "bad density arguments");
  RSED_REQUIRE(n_density == 0 || (dens_i && dens_j && dens_v), RSED_EINVAL, "density terms missing");
  cudaStream_t stream = as_stream(stream_);
  k_density_diag<<<(unsigned)((n_orbits + 255) / 256), 256, 0, stream>>>(
      n_orbits, repr_masks, n_density, dens_i, dens_j, reinterpret_cast<const double2*>(dens_v),
      reinterpret_cast<double2*>(hdiag));
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}

// ---- sector rows without device allocation ----------------------------------
// rsed_sector_rows_noalloc: the same result as rsed_sector_rows, for callers
// that cannot hand the library a scratch buffer.  Its only scratch is the
// per-tile sums of the scan, held in this file-scope device array (one copy
// on every GPU that loads the library, kept until the process exits).  The
// member bit is re-derived from `member` in both passes instead of being
// stored, so no buffer proportional to n_orbits is needed.
namespace {

constexpr int64_t kNoAllocMaxTiles = 16384;  // 16384 tiles x 8192 orbits = 2^27 orbits
constexpr int64_t kNoAllocMaxOrbits = kNoAllocMaxTiles * kScanTile;

// tile sums (kNoAllocMaxTiles) followed by the total
static __device__ __align__(256) int64_t g_rows_scan_scratch[kNoAllocMaxTiles + 1];

__global__ void k_nb_tile_counts(int64_t n, const uint64_t* member, int sector, int64_t* tile_sum) {
  __shared__ int64_t tot;
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int64_t c = 0;
  for (int j = 0; j < kScanItems; ++j) {
    const int64_t i = base + j;
    if (i < n) c += (member[i] >> sector) & 1ull;
  }
  block_exclusive_scan(c, &tot);
  if (threadIdx.x == 0) tile_sum[blockIdx.x] = tot;
}

__global__ void k_nb_tile_rows(int64_t n, const uint64_t* member, int sector, const int64_t* tile_off,
                               int32_t* orbit_of_row, int32_t* row_of_orbit) {
  __shared__ int64_t tot;
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int flag[kScanItems];
  int64_t c = 0;
  for (int j = 0; j < kScanItems; ++j) {
    const int64_t i = base + j;
    flag[j] = (i < n) ? (int)((member[i] >> sector) & 1ull) : 0;
    c += flag[j];
  }
  int64_t pos = block_exclusive_scan(c, &tot) + tile_off[blockIdx.x];
  for (int j = 0; j < kScanItems; ++j) {
    const int64_t i = base + j;
    if (i >= n) break;
    if (flag[j]) {
      if (orbit_of_row) orbit_of_row[pos] = (int32_t)i;
      if (row_of_orbit) row_of_orbit[i] = (int32_t)pos;
      ++pos;
    } else if (row_of_orbit) {
      row_of_orbit[i] = -1;
    }
  }
}

// Device address of the scratch array, looked up once per device.
std::mutex g_noalloc_mu;
int64_t* g_noalloc_ptr[64] = {nullptr};

int noalloc_scratch(int64_t** out) {
  int dev = -1;
  RSED_TRY_CUDA(cudaGetDevice(&dev));
  RSED_REQUIRE(dev >= 0 && dev < 64, RSED_ERANGE, "device ordinal %d outside [0, 64)", dev);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (g_noalloc_ptr[dev] == nullptr) {
    void* p = nullptr;
    RSED_TRY_CUDA(cudaGetSymbolAddress(&p, g_rows_scan_scratch));
    g_noalloc_ptr[dev] = reinterpret_cast<int64_t*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return RSED_OK;
}

}  // namespace

extern "C" int rsed_sector_rows_noalloc(int64_t n_orbits, const uint64_t* member, int32_t sector,
                                        int32_t* orbit_of_row, int32_t* row_of_orbit, void* stream_) {
  RSED_REQUIRE(n_orbits >= 1 && member && sector >= 0 && sector < 64, RSED_EINVAL,
               "bad sector-rows arguments");
  RSED_REQUIRE(orbit_of_row || row_of_orbit, RSED_EINVAL, "no output buffer");
  RSED_REQUIRE(n_orbits <= kNoAllocMaxOrbits, RSED_ERANGE,
               "rsed_sector_rows_noalloc handles at most %lld orbits (got %lld); "
               "use rsed_sector_rows with a caller-owned scratch buffer",
               (long long)kNoAllocMaxOrbits, (long long)n_orbits);
  int64_t* scratch = nullptr;
  int rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  cudaStream_t stream = as_stream(stream_);
  const int64_t tiles = (n_orbits + kScanTile - 1) / kScanTile;
  int64_t* tile_sum = scratch;
  int64_t* total = scratch + kNoAllocMaxTiles;
  // every tile sum and the total are rewritten below, so the contents left
  // by an earlier call need no clearing
  k_nb_tile_counts<<<(unsigned)tiles, kScanThreads, 0, stream>>>(n_orbits, member, sector, tile_sum);
  RSED_CHECK_LAUNCH();
  k_scan_tiles<<<1, kScanThreads, 0, stream>>>(tile_sum, tiles, total);
  RSED_CHECK_LAUNCH();
  k_nb_tile_rows<<<(unsigned)tiles, kScanThreads, 0, stream>>>(n_orbits, member, sector, tile_sum,
                                                               orbit_of_row, row_of_orbit);
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}

extern "C" int64_t rsed_sector_rows_noalloc_max_orbits(void) { return kNoAllocMaxOrbits; }
