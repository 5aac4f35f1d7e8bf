// Correlators of one sector state: the one-body density matrix
// rho[i][j] = <psi| a_i^dagger a_j |psi> (off_diagonal_long_range_order,
// observables/off_diagonal_long_range_order.py:43-140) and the orbit-summed
// density pairs behind the static structure factor
// (_build_density_correlation_matrix, observables/static_structure_factor.py:54-149).
//
// Both reduce over the orbits of a sector into an N x N matrix.  Every matrix
// entry is owned by one thread of a block, accumulated in shared memory in a
// fixed order (no atomics); one wave of blocks walks the orbit chunks with a
// grid stride, writes one partial matrix per block, and a final pass adds the
// block partials in block order -- the same sums on every run of a device.
#include "rsed_internal.cuh"

namespace {

constexpr int kCT = 256;

int one_wave(const void* fn, size_t smem) {
  int dev = 0, n_sm = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -1;
  if (cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kCT, smem) != cudaSuccess) return -1;
  return n_sm * (per_sm > 0 ? per_sm : 1);
}

// ---- one-body density matrix ------------------------------------------------
//
// For an orbit o (representative s, coefficient c_o != 0) and group element g,
// the ket |g s> carries c_o / sqrt(|G| |Stab(s)|) * conj(chi(g)) * phase_g(s).
// rho[j][j] gains |c_o|^2 / |G| for every occupied j; for an empty i the hop
// j -> i lands on a mask whose canonical entry (rep', g', alpha') names the
// bra: c_rep' * sqrt(|Stab(rep')| / |G|) * conj(alpha' conj(chi(g'))), if rep'
// is in the sector; rho[i][j] += conj(bra) * ket * (Jordan-Wigner sign of the
// hop for fermions).  Kets are staged kCT at a time in shared memory (a chunk
// of kCT / |G| orbits); each thread then walks the staged kets for the (i, j)
// entries it owns.
struct Ket {
  uint64_t mask;
  double2 amp;
  double diag;
};

__global__ void __launch_bounds__(kCT) k_obdm_part(rsed_group_t grp, const int4* __restrict__ table,
                                                   int64_t n_orbits, const uint64_t* __restrict__ repr_masks,
                                                   const uint64_t* __restrict__ stab_mask,
                                                   const uint64_t* __restrict__ member, int sector,
                                                   const double2* __restrict__ chi, const double2* __restrict__ x,
                                                   double2* __restrict__ part) {
  extern __shared__ double2 acc[];  // N*N owner-written accumulators
  __shared__ Ket kets[kCT];
  const int N = grp.n_site;
  const int NN = N * N;
  const int ng = grp.n_group;
  const int per_chunk = kCT / ng;  // orbits per chunk (|G| <= 64)
  const int64_t n_chunks = (n_orbits + per_chunk - 1) / per_chunk;
  const int kp1 = grp.n_filled + 1;
  const bool fermion = grp.fermionic != 0;
  const double2* eta = reinterpret_cast<const double2*>(grp.eta);
  const double inv_sqrt_ng = 1.0 / sqrt((double)ng);
  const double inv_ng = 1.0 / (double)ng;
  const uint64_t sbit = 1ull << sector;
  int64_t cb = 0;
  if (grp.species_b) {
    const RsedSpecies sp = rsed_species(grp.species_b, N, grp.n_filled, grp.n_filled_b, grp.binom, kp1);
    cb = sp.cb;
  }
  for (int p = threadIdx.x; p < NN; p += kCT) acc[p] = make_double2(0.0, 0.0);
  for (int64_t ch = blockIdx.x; ch < n_chunks; ch += gridDim.x) {
    __syncthreads();  // the previous chunk's kets are consumed
    {
      const int t = threadIdx.x;
      Ket k;
      k.mask = 0;
      k.amp = make_double2(0.0, 0.0);
      k.diag = 0.0;
      const int64_t o = ch * per_chunk + t / ng;
      if (t < per_chunk * ng && o < n_orbits) {
        const double2 c = x[o];
        if (c.x != 0.0 || c.y != 0.0) {
          const int g = t % ng;
          const uint64_t s = repr_masks[o];
          uint64_t img;
          const double2 ph = rsed_phase_product(s, grp.perm + (int64_t)g * N, eta + (int64_t)g * N, fermion, &img);
          const double norm = inv_sqrt_ng / sqrt((double)__popcll(stab_mask[o]));
          const double2 cg = make_double2(chi[g].x, -chi[g].y);
          const double2 basis_amp = cmul(make_double2(norm * cg.x, norm * cg.y), ph);
          k.mask = img;
          k.amp = cmul(c, basis_amp);
          k.diag = (c.x * c.x + c.y * c.y) * inv_ng;
        }
      }
      kets[t] = k;
    }
    __syncthreads();
    for (int p = threadIdx.x; p < NN; p += kCT) {
      const int i = p / N, j = p % N;
      double2 a = acc[p];
      for (int q = 0; q < kCT; ++q) {
        const uint64_t m = kets[q].mask;
        if (!((m >> j) & 1ull)) continue;  // j must be occupied (also skips empty slots)
        if (i == j) {
          a.x += kets[q].diag;
          continue;
        }
        if ((m >> i) & 1ull) continue;  // i must be empty
        // a hop between the species of a two-species basis leaves the basis: zero
        if (((grp.species_b >> i) ^ (grp.species_b >> j)) & 1ull) continue;
        const uint64_t nm = m ^ (1ull << j) ^ (1ull << i);
        const int64_t r = rsed_rank_any(nm, grp.binom, kp1, grp.species_b, cb);
        if (r < 0 || r >= grp.n_states) continue;
        const int4 e = __ldg(table + r);
        if (e.x < 0 || !(member[e.x] & sbit)) continue;
        const double2 cr = x[e.x];
        const double2 alpha = make_double2((double)__int_as_float(e.z), (double)__int_as_float(e.w));
        const double2 pc = cmul(alpha, make_double2(chi[e.y].x, -chi[e.y].y));
        const double sr = sqrt((double)__popcll(stab_mask[e.x])) * inv_sqrt_ng;
        const double2 bra = cmul(cr, make_double2(sr * pc.x, -sr * pc.y));
        double2 t = cmul(make_double2(bra.x, -bra.y), kets[q].amp);
        if (fermion) {
          const int lo = min(i, j), hi = max(i, j);
          const uint64_t between = (hi - lo > 1) ? (((1ull << (hi - lo - 1)) - 1ull) << (lo + 1)) : 0ull;
          if (__popcll(m & between) & 1) t = make_double2(-t.x, -t.y);
        }
        a.x += t.x;
        a.y += t.y;
      }
      acc[p] = a;
    }
  }
  __syncthreads();
  for (int p = threadIdx.x; p < NN; p += kCT) part[(int64_t)blockIdx.x * NN + p] = acc[p];
}

// ---- density pairs --------------------------------------------------------------
//
// D[a][b] = sum_o |x_o|^2 n_a(s_o) n_b(s_o) over the representatives s_o; the
// structure factor's C[i][j] = (1/|G|) sum_g D[a][b] at i = g(a), j = g(b)
// follows from it on the host.
__global__ void __launch_bounds__(kCT) k_pairs_part(int n_site, int64_t n_orbits,
                                                    const uint64_t* __restrict__ repr_masks,
                                                    const double2* __restrict__ x, double* __restrict__ part) {
  extern __shared__ double dacc[];
  __shared__ uint64_t sm[kCT];
  __shared__ double sw[kCT];
  const int N = n_site, NN = N * N;
  const int64_t n_chunks = (n_orbits + kCT - 1) / kCT;
  for (int p = threadIdx.x; p < NN; p += kCT) dacc[p] = 0.0;
  for (int64_t ch = blockIdx.x; ch < n_chunks; ch += gridDim.x) {
    __syncthreads();
    const int64_t o = ch * kCT + threadIdx.x;
    if (o < n_orbits) {
      const double2 c = x[o];
      sm[threadIdx.x] = repr_masks[o];
      sw[threadIdx.x] = c.x * c.x + c.y * c.y;
    } else {
      sm[threadIdx.x] = 0;
      sw[threadIdx.x] = 0.0;
    }
    __syncthreads();
    for (int p = threadIdx.x; p < NN; p += kCT) {
      const uint64_t both = (1ull << (p / N)) | (1ull << (p % N));
      double d = dacc[p];
      for (int q = 0; q < kCT; ++q)
        if ((sm[q] & both) == both) d += sw[q];
      dacc[p] = d;
    }
  }
  __syncthreads();
  for (int p = threadIdx.x; p < NN; p += kCT) part[(int64_t)blockIdx.x * NN + p] = dacc[p];
}

template <typename T>
__global__ void k_sum_blocks(const T* __restrict__ part, int n_blocks, int nn, T* __restrict__ out);

template <>
__global__ void k_sum_blocks<double2>(const double2* __restrict__ part, int n_blocks, int nn,
                                      double2* __restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nn) return;
  double2 s = make_double2(0.0, 0.0);
  for (int b = 0; b < n_blocks; ++b) {
    const double2 v = part[(int64_t)b * nn + p];
    s.x += v.x;
    s.y += v.y;
  }
  out[p] = s;
}

template <>
__global__ void k_sum_blocks<double>(const double* __restrict__ part, int n_blocks, int nn, double* __restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nn) return;
  double s = 0.0;
  for (int b = 0; b < n_blocks; ++b) s += part[(int64_t)b * nn + p];
  out[p] = s;
}

int obdm_grid(int n_site, size_t* smem) {
  *smem = sizeof(double2) * (size_t)n_site * n_site;
  if (*smem > 48 * 1024 &&
      cudaFuncSetAttribute(k_obdm_part, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem) != cudaSuccess)
    return -1;
  return one_wave((const void*)k_obdm_part, *smem);
}

int pairs_grid(int n_site, size_t* smem) {
  *smem = sizeof(double) * (size_t)n_site * n_site;
  return one_wave((const void*)k_pairs_part, *smem);
}

}  // namespace

extern "C" size_t rsed_obdm_scratch_bytes(int32_t n_site) {
  size_t smem = 0;
  const int grid = obdm_grid(n_site, &smem);
  if (grid <= 0) return 0;
  return sizeof(double2) * (size_t)grid * n_site * n_site;
}

extern "C" int rsed_one_body_density(const rsed_group_t* grp, const rsed_entry_t* table, int64_t n_orbits,
                                     const uint64_t* repr_masks, const uint64_t* stab_mask, const uint64_t* member,
                                     int32_t sector, const double* chi, const double* x_orbit, double* rho,
                                     void* scratch, size_t scratch_bytes, void* stream_) {
  int rc = check_group(grp);
  if (rc) return rc;
  RSED_REQUIRE(table && repr_masks && stab_mask && member && chi && x_orbit && rho && scratch && n_orbits >= 1,
               RSED_EINVAL, "bad one-body density arguments");
  RSED_REQUIRE(grp->eta != nullptr, RSED_EINVAL, "one-body density needs the group's eta phases");
  RSED_REQUIRE(sector >= 0 && sector < 64, RSED_EINVAL, "sector index %d outside [0, 64)", sector);
  size_t smem = 0;
  const int grid = obdm_grid(grp->n_site, &smem);
  RSED_REQUIRE(grid > 0, RSED_ECUDA, "no occupancy for the one-body density kernel");
  RSED_REQUIRE(scratch_bytes >= sizeof(double2) * (size_t)grid * grp->n_site * grp->n_site, RSED_ESCRATCH,
               "one-body density scratch too small");
  cudaStream_t stream = as_stream(stream_);
  double2* part = reinterpret_cast<double2*>(scratch);
  k_obdm_part<<<grid, kCT, smem, stream>>>(*grp, reinterpret_cast<const int4*>(table), n_orbits, repr_masks,
                                          stab_mask, member, sector, reinterpret_cast<const double2*>(chi),
                                          reinterpret_cast<const double2*>(x_orbit), part);
  RSED_CHECK_LAUNCH();
  const int nn = grp->n_site * grp->n_site;
  k_sum_blocks<double2><<<(nn + 127) / 128, 128, 0, stream>>>(part, grid, nn, reinterpret_cast<double2*>(rho));
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}

extern "C" size_t rsed_density_pairs_scratch_bytes(int32_t n_site) {
  size_t smem = 0;
  const int grid = pairs_grid(n_site, &smem);
  if (grid <= 0) return 0;
  return sizeof(double) * (size_t)grid * n_site * n_site;
}

extern "C" int rsed_density_pairs(int32_t n_site, int64_t n_orbits, const uint64_t* repr_masks,
                                  const double* x_orbit, double* pairs, void* scratch, size_t scratch_bytes,
                                  void* stream_) {
  RSED_REQUIRE(n_site >= 1 && n_site <= RSED_MAX_SITES, RSED_ERANGE, "n_site = %d outside [1, %d]", n_site,
               RSED_MAX_SITES);
  RSED_REQUIRE(repr_masks && x_orbit && pairs && scratch && n_orbits >= 1, RSED_EINVAL,
               "bad density-pair arguments");
  size_t smem = 0;
  const int grid = pairs_grid(n_site, &smem);
  RSED_REQUIRE(grid > 0, RSED_ECUDA, "no occupancy for the density-pair kernel");
  RSED_REQUIRE(scratch_bytes >= sizeof(double) * (size_t)grid * n_site * n_site, RSED_ESCRATCH,
               "density-pair scratch too small");
  cudaStream_t stream = as_stream(stream_);
  double* part = reinterpret_cast<double*>(scratch);
  k_pairs_part<<<grid, kCT, smem, stream>>>(n_site, n_orbits, repr_masks, reinterpret_cast<const double2*>(x_orbit),
                                           part);
  RSED_CHECK_LAUNCH();
  const int nn = n_site * n_site;
  k_sum_blocks<double><<<(nn + 127) / 128, 128, 0, stream>>>(part, grid, nn, pairs);
  RSED_CHECK_LAUNCH();
  return RSED_OK;
}
