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
