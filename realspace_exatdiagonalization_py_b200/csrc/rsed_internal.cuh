// Host-side helpers shared by the .cu translation units of librsed.so.
#pragma once
#include <cstdarg>
#include <cstdio>
#include <string>
#include "rsed_common.cuh"

int rsed_set_error(int code, const char* fmt, ...);
// Number of kernels this library has launched (all host threads).
void rsed_count_launch();

#define RSED_TRY_CUDA(expr)                                                      \
  do {                                                                           \
    cudaError_t _e = (expr);                                                     \
    if (_e != cudaSuccess)                                                       \
      return rsed_set_error(RSED_ECUDA, "%s: %s (%s:%d)", #expr,                 \
                            cudaGetErrorString(_e), __FILE__, __LINE__);         \
  } while (0)

#define RSED_CHECK_LAUNCH()                                                      \
  do {                                                                           \
    rsed_count_launch();                                                         \
    cudaError_t _e = cudaGetLastError();                                         \
    if (_e != cudaSuccess)                                                       \
      return rsed_set_error(RSED_ECUDA, "kernel launch: %s (%s:%d)",             \
                            cudaGetErrorString(_e), __FILE__, __LINE__);         \
  } while (0)

#define RSED_REQUIRE(cond, code, ...)                                            \
  do {                                                                           \
    if (!(cond)) return rsed_set_error(code, __VA_ARGS__);                       \
  } while (0)

static inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

static inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Exclusive scan of n int64 counts into out[0..n] (out[n] = total), on
// `stream`.  Needs rsed_scan_scratch_bytes(n) bytes of scratch.
size_t rsed_scan_scratch_bytes(int64_t n);
int rsed_exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t n, void* scratch,
                            size_t scratch_bytes, cudaStream_t stream);

// Bytes of dynamic shared memory used to stage a group (binomials, perms,
// angles, eta) in catalog-type kernels.
struct GroupSmemLayout {
  size_t binom_off, perm_off, angle_off, eta_off, total;
};
GroupSmemLayout group_smem_layout(int n_site, int n_filled, int n_group, bool with_eta,
                                  bool with_angle);
int check_group(const rsed_group_t* g);
// Streaming apply over the model's projection table (proj.cu); variant 0
// picks the column chunk, 3NN / 4NN as documented at rsed_apply_h.
int rsed_proj_apply(const rsed_model_t& md, const rsed_sectors_t& sc, const void* x, double2* y, int precision,
                    int variant, cudaStream_t stream);
