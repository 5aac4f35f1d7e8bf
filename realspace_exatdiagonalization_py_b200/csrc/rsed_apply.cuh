// Shared-memory staging of a Hamiltonian's term tables and the 16-B table
// load used by the matrix-free apply (apply.cu) and the persistent Lanczos
// kernel (lanczos.cu).
#pragma once
#include "rsed_internal.cuh"

namespace rsed_apply {

struct ApplySmemLayout {
  size_t binom, tbeg, tto, tamp, tjw, chi, csec, total;
};

inline ApplySmemLayout apply_layout(const rsed_model_t& md, const rsed_sectors_t& sc) {
  ApplySmemLayout l{};
  size_t off = 0;
  l.tamp = off;
  off = align_up(off + sizeof(double2) * md.n_terms, 16);
  l.chi = off;
  off = align_up(off + sizeof(double2) * (size_t)sc.n_sectors * md.n_group, 16);
  l.binom = off;
  off = align_up(off + sizeof(int64_t) * (size_t)(md.n_site + 1) * (md.n_filled + 1), 16);
  l.tjw = off;
  off = align_up(off + sizeof(uint64_t) * md.n_terms, 16);
  l.tbeg = off;
  off = align_up(off + sizeof(int32_t) * (md.n_site + 1), 16);
  l.csec = off;
  off = align_up(off + sizeof(int32_t) * sc.n_cols, 16);
  l.tto = off;
  off = align_up(off + (size_t)md.n_terms, 16);
  l.total = off;
  return l;
}

struct ApplyView {
  const int64_t* binom;
  const int32_t* tbeg;
  const uint8_t* tto;
  const double2* tamp;
  const uint64_t* tjw;
  const double2* chi;
  const int32_t* csec;
};

__device__ inline ApplyView stage_apply(const rsed_model_t& md, const rsed_sectors_t& sc,
                                 const ApplySmemLayout& l, unsigned char* smem) {
  ApplyView v;
  int64_t* b = reinterpret_cast<int64_t*>(smem + l.binom);
  int nb = (md.n_site + 1) * (md.n_filled + 1);
  for (int i = threadIdx.x; i < nb; i += blockDim.x) b[i] = md.binom[i];
  int32_t* tb = reinterpret_cast<int32_t*>(smem + l.tbeg);
  for (int i = threadIdx.x; i <= md.n_site; i += blockDim.x) tb[i] = md.term_begin[i];
  uint8_t* tt = smem + l.tto;
  double2* ta = reinterpret_cast<double2*>(smem + l.tamp);
  uint64_t* tj = reinterpret_cast<uint64_t*>(smem + l.tjw);
  const double2* gamp = reinterpret_cast<const double2*>(md.term_amp);
  for (int i = threadIdx.x; i < md.n_terms; i += blockDim.x) {
    tt[i] = md.term_to[i];
    ta[i] = gamp[i];
    tj[i] = md.term_jw[i];
  }
  double2* ch = reinterpret_cast<double2*>(smem + l.chi);
  const double2* gchi = reinterpret_cast<const double2*>(sc.chi);
  for (int i = threadIdx.x; i < sc.n_sectors * md.n_group; i += blockDim.x) ch[i] = gchi[i];
  int32_t* cs = reinterpret_cast<int32_t*>(smem + l.csec);
  for (int i = threadIdx.x; i < sc.n_cols; i += blockDim.x) cs[i] = sc.col_sector[i];
  __syncthreads();
  v.binom = b;
  v.tbeg = tb;
  v.tto = tt;
  v.tamp = ta;
  v.tjw = tj;
  v.chi = ch;
  v.csec = cs;
  return v;
}

__device__ __forceinline__ RsedEntry load_entry(const RsedEntry* t, int64_t idx) {
  int4 r = __ldg(reinterpret_cast<const int4*>(t) + idx);
  RsedEntry e;
  e.rep = r.x;
  e.g = r.y;
  e.re = __int_as_float(r.z);
  e.im = __int_as_float(r.w);
  return e;
}

}  // namespace rsed_apply
