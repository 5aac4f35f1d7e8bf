/*
 * rsed.h — C ABI of the B200 symmetry-resolved exact-diagonalization library
 * (librsed.so, sm_100a).
 *
 * Every entry point takes plain device pointers, sizes and a cudaStream_t
 * passed as `void*` (NULL = legacy default stream), returns 0 on success or a
 * negative RSED_E* code, and never allocates device memory: scratch buffers
 * are sized by the matching *_scratch_bytes() query and owned by the caller.
 * Complex numbers are interleaved (re, im) pairs of double (complex128) or
 * float (complex64).  Sites are 0-based inside the ABI (the reference's
 * 1-based site i is bit i-1).
 *
 * The reference (realspace_exactdiagonalization_py) has no FFI layer: its
 * hot path is the set of Python functions in
 * src/realspace_exactdiagonalization_py/symmetry_resolved_ed.py.  Each entry
 * point below names the reference function (file:line) it replaces; the
 * Python binding that calls it is
 * realspace_exatdiagonalization_py_b200/_lib.py (ctypes).
 */
#ifndef RSED_H_
#define RSED_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RSED_OK 0
#define RSED_EINVAL -1      /* bad argument (maps to ValueError / AssertionError) */
#define RSED_ECUDA -2       /* CUDA runtime error (launch or execution) */
#define RSED_ENOTCONV -3    /* eigensolver hit its iteration cap */
#define RSED_ERANGE -4      /* size beyond a compiled or documented limit */
#define RSED_EBREAKDOWN -5  /* Krylov block lost rank (Cholesky pivot <= 0) */
#define RSED_ESCRATCH -6    /* scratch buffer smaller than the query returned */
#define RSED_ETIMEOUT -7    /* a device-side wait ran past its time limit (no result written) */

/* One representative-table entry (16 bytes), indexed by combinadic rank:
 * the reference's rep_rank_table / rep_sym_table / rep_amp_table
 * (symmetry_resolved_ed.py:1359-1361) interleaved per state. */
typedef struct {
  int32_t rep;  /* 0-based orbit (representative) index */
  int32_t g;    /* 0-based group element with g(rep) = mask */
  float re, im; /* complex64 canonicalisation amplitude alpha_g(rep) */
} rsed_entry_t;

/* Symmetry group of a catalog (device pointers). */
typedef struct {
  int32_t n_site;      /* N <= 63 */
  int32_t n_filled;    /* k, 0 <= k <= N */
  int32_t n_group;     /* |G| <= 64 */
  int32_t fermionic;   /* 1 = fermions (permutation parity), 0 = hard-core bosons */
  int64_t n_states;    /* C(N, k) */
  const int64_t* binom; /* (N+1) x (k+1) row-major, C(b, j) */
  const uint8_t* perm;  /* |G| x N: 0-based image site of site i under g */
  const double* angle;  /* |G| x N: numpy.angle(eta_g(i)) */
  const double* eta;    /* |G| x N complex128: eta_g(i) */
  /* Two-species bases (particle number fixed per species, e.g. per spin):
   * species_b marks the sites of species B, which hold n_filled_b of the
   * n_filled particles; 0 = one species.  States are ranked
   * rank_A * C(|B|, n_filled_b) + rank_B, each species in colex order over its
   * own sites; n_states = C(N - |B|, n_filled - n_filled_b) * C(|B|, n_filled_b).
   * Every group element must map species B onto itself. */
  uint64_t species_b;
  int32_t n_filled_b;
  int32_t reserved_b;
} rsed_group_t;

/* Hopping / density model on the orbit basis of one catalog. */
typedef struct {
  int32_t n_site, n_filled, n_group, fermionic;
  int64_t n_states;
  int64_t n_orbits;
  const int64_t* binom;          /* as in rsed_group_t */
  const rsed_entry_t* table;     /* n_states entries */
  const uint64_t* repr_masks;    /* n_orbits representative masks (ascending) */
  int32_t n_terms;               /* directed bilinear terms after merging duplicates */
  const int32_t* term_begin;     /* N+1: terms grouped by annihilated (source) site */
  const uint8_t* term_to;        /* n_terms: created (target) site */
  const double* term_amp;        /* n_terms complex128 amplitudes */
  const uint64_t* term_jw;       /* n_terms: sites strictly between source and target */
  const double* hdiag;           /* n_orbits complex128 density-density diagonal */
  /* Optional orbit-space projection table (rsed_proj_fill); proj_rowptr NULL
   * = none.  When present, rsed_apply_h streams it instead of re-deriving
   * every hop (variants 0 and 3xx/4xx). */
  const int64_t* proj_rowptr;    /* n_orbits + 1 entry offsets */
  const uint32_t* proj_cg;       /* per hop: target orbit | g << 26 */
  const double* proj_w64;        /* per hop complex128 weight, or NULL */
  const float* proj_w32;         /* per hop complex64 weight, or NULL */
  uint64_t species_b;            /* as in rsed_group_t */
  int32_t n_filled_b;
  int32_t reserved_b;
} rsed_model_t;

/* A set of momentum sectors evaluated together ("columns" of a block of
 * vectors laid out row-major as [n_orbits][ld], one row per orbit). */
typedef struct {
  int32_t n_sectors;          /* <= 64 */
  int32_t n_cols;             /* columns in use */
  int32_t ld;                 /* leading dimension (elements) >= n_cols */
  int32_t n_group;
  const uint64_t* member;     /* n_orbits: bit s set if the orbit belongs to sector s */
  const double* sqrt_stab;    /* n_orbits: sqrt(|Stab|) */
  const double* chi;          /* n_sectors x n_group complex128 characters */
  const int32_t* col_sector;  /* n_cols: sector of each column */
} rsed_sectors_t;

const char* rsed_version(void);
/* Message of the last error raised on the calling host thread. */
const char* rsed_last_error(void);

/* ---- K1-K3: orbit catalog -------------------------------------------------
 * Replaces build_symmetry_orbit_catalog / _build_orbit_catalog_kernel
 * (symmetry_resolved_ed.py:1298-1404, 433-575).  The caller allocates the
 * outputs once the counts are known, hence the call sequence
 *   rsed_catalog_count   representative test over all C(N,k) states -> *n_orbits_out
 *   rsed_catalog_fill    representative masks (rank order), the whole table
 *                        (g = 0..|G|-1 written in ascending g so the last writer
 *                        wins, as the reference does) and stabilizer bitmasks
 *   rsed_catalog_stab_count  exclusive stabilizer offsets -> *n_stab_out
 *   rsed_catalog_stab    complex128 stabilizer phases, ascending g per orbit.
 * The scratch of rsed_catalog_count must be passed unchanged to _fill. */
size_t rsed_catalog_scratch_bytes(const rsed_group_t* grp);
int rsed_catalog_count(const rsed_group_t* grp, void* scratch, size_t scratch_bytes,
                       int64_t* n_orbits_out, void* stream);
int rsed_catalog_fill(const rsed_group_t* grp, const void* scratch, size_t scratch_bytes,
                      int64_t n_orbits, uint64_t* repr_masks, rsed_entry_t* table,
                      uint64_t* stab_mask, void* stream);
size_t rsed_stab_scratch_bytes(int64_t n_orbits);
int rsed_catalog_stab_count(int64_t n_orbits, const uint64_t* stab_mask, int64_t* stab_off,
                            int64_t* n_stab_out, void* scratch, size_t scratch_bytes, void* stream);
int rsed_catalog_stab(const rsed_group_t* grp, int64_t n_orbits, const uint64_t* repr_masks,
                      const uint64_t* stab_mask, const int64_t* stab_off, double* stab_phase,
                      void* stream);

/* ---- K4: flux phase update ------------------------------------------------
 * Replaces update_orbit_stabilizer_phases (symmetry_resolved_ed.py:1220-1269):
 * recompute the stabilizer phases and rewrite g / alpha of every table entry
 * for a group with the same permutations and new per-site phases (product
 * form, ascending g, last writer wins).  In place.  *err_dev (device int)
 * becomes non-zero if the catalog does not match the group. */
int rsed_phase_update(const rsed_group_t* grp, int64_t n_orbits, const uint64_t* repr_masks,
                      const uint64_t* stab_mask, const int64_t* stab_off, double* stab_phase,
                      rsed_entry_t* table, int* err_dev, void* stream);

/* ---- K5: sector membership ----------------------------------------------
 * Replaces _is_orbit_compatible / build_symmetry_sector_basis
 * (symmetry_resolved_ed.py:1484-1546) for many irreps at once: bit s of
 * member[o] is set iff |chi_s(h) - alpha_h| <= atol for every h in Stab(o).
 * sqrt_stab[o] = sqrt(popcount(stab_mask[o])).  sector_dims[s] (device
 * int64) receives the dimension of sector s. */
int rsed_sector_members(int64_t n_orbits, int32_t n_group, int32_t n_sectors,
                        const uint64_t* stab_mask, const int64_t* stab_off,
                        const double* stab_phase, const double* chi, double atol,
                        uint64_t* member, double* sqrt_stab, int64_t* sector_dims, void* stream);
/* Basis of one sector (the reference's Symmetry_Sector_Basis order): orbit of
 * each basis row (ascending) and the row of each orbit (-1 if absent). */
size_t rsed_sector_scratch_bytes(int64_t n_orbits, int32_t n_sectors);
int rsed_sector_rows(int64_t n_orbits, const uint64_t* member, int32_t sector,
                     int32_t* orbit_of_row, int32_t* row_of_orbit, void* scratch,
                     size_t scratch_bytes, void* stream);

/* Same output as rsed_sector_rows, without any caller scratch: for callers
 * that cannot allocate device memory -- services that reserve the GPU's
 * memory up front in their own pool and forbid later allocations, and
 * latency-critical loops that must not hit the device-wide synchronisation
 * that cudaFree performs.  No counterpart in the reference (it has no C
 * interface at all).  The scan's tile sums live in a file-scope __device__
 * array sized for at most rsed_sector_rows_noalloc_max_orbits() = 2^27 orbits
 * (128 KiB, present on every GPU that loads the library until the process
 * exits); larger inputs return RSED_ERANGE.  The array's device address is
 * looked up on the first call on each device, so make that first call before
 * any stream capture.  All calls share the array: calls that can overlap on
 * the GPU (different streams, different host threads) race and must be
 * serialised by the caller.  It calls no cudaMalloc/cudaFree. */
int rsed_sector_rows_noalloc(int64_t n_orbits, const uint64_t* member, int32_t sector,
                             int32_t* orbit_of_row, int32_t* row_of_orbit, void* stream);
int64_t rsed_sector_rows_noalloc_max_orbits(void);

/* Density-density diagonal per orbit, summed in term order like the
 * reference's h_diag (symmetry_resolved_ed.py:641-646). */
int rsed_density_diag(int64_t n_orbits, const uint64_t* repr_masks, int32_t n_density,
                      const uint8_t* dens_i, const uint8_t* dens_j, const double* dens_v,
                      double* hdiag, void* stream);

/* ---- K6: matrix-free H|psi> ------------------------------------------------
 * Replaces MatrixFreeHamiltonian.__call__ / _apply_hamiltonian_kernel
 * (symmetry_resolved_ed.py:1965-1976, 826-923) for all columns of a block at
 * once.  Pull form without atomics: row r of a column accumulates
 * conj(H[s, r]) x[s] over the hops from rep(r), i.e. y = H^dagger x, which is
 * H x for the Hermitian blocks the reference builds (to the complex64
 * rounding of its amplitude table).  precision 64: x complex128, FP64
 * accumulation; precision 32: x complex64, FP32 accumulation; y is always
 * complex128.  variant 0 streams the model's projection table when it has one
 * (K6b below) and otherwise picks the on-the-fly lane mapping from n_cols;
 * 999 always picks the on-the-fly mapping; 1..299 name one on-the-fly
 * mapping. */
int rsed_apply_h(const rsed_model_t* model, const rsed_sectors_t* sec, const void* x, void* y,
                 int32_t precision, int32_t variant, void* stream);

/* ---- K6b: orbit-space projection table ---------------------------------
 * The sector-independent part of every hop of every orbit row, built once per
 * catalog state (the device form of build_matrixfree_projection_table /
 * _build_matrixfree_table_kernel, symmetry_resolved_ed.py:1719-1769, 751-799,
 * shared by all sectors instead of one table per sector).  Row r holds, in the
 * hop order of rsed_apply_h (occupied source site ascending, then term order),
 *   cg = c | g << 26     target orbit c, group element g of the table entry
 *   w  = conj(t * s_JW * alpha) * sqrt(S_c) / sqrt(S_r)
 * so that column j of y = H^dagger x gets sum_hops w * chi_s(g) * x[c][j]
 * (s = sector of column j) plus conj(h_diag[r]) x[r][j].  Needs n_orbits <
 * 2^26 and |G| <= 64.  rsed_proj_count writes rowptr (n_orbits + 1) and the
 * number of hops; rsed_proj_fill writes cg and either weight array (each
 * NULL = skip: cg is the same for every amplitude update of one catalog, so
 * tables of several flux points can share one cg and rowptr).  With the table set in the model, rsed_apply_h variant 3NN streams
 * it over column chunks of NN columns one chunk after another (the chunk of x
 * stays in L2 while the table streams from HBM), 4NN runs all chunks in one
 * launch; NN in {2,4,8,16,32} at precision 64 and {4,8,16,32,64} at 32.
 * 5NN / 6NN are the same with a 32-B instead of a 16-B segment of x per lane
 * and hop; NN in {4,8,16,32,64} at precision 64 and {8,16,32,64} at 32, and
 * 528 / 628 for 128 columns at precision 32.
 * These variants read x only at rows of the column's sector: rows outside it
 * must hold zero (the Lanczos buffers keep them zero). */
size_t rsed_proj_scratch_bytes(int64_t n_orbits);
int rsed_proj_count(const rsed_model_t* model, int64_t* rowptr, int64_t* n_hops_out, void* scratch,
                    size_t scratch_bytes, void* stream);
int rsed_proj_fill(const rsed_model_t* model, const double* sqrt_stab, const int64_t* rowptr,
                   uint32_t* cg, double* w64, float* w32, void* stream);

/* ---- K7: matrix mode ---------------------------------------------------
 * Replaces _vectorized_block_triplets / _build_H_block_kernel
 * (symmetry_resolved_ed.py:595-736): exact (row, col, value) triplets of one
 * sector block, value ((((t * s_JW) * alpha) * conj(chi(g))) * sqrt(S_row/S_col))
 * in the reference's product order, diagonal first per column.  count fills
 * col_off (n_rows+1 exclusive offsets) and *nnz_out; fill writes the triplets. */
size_t rsed_triplet_scratch_bytes(int64_t n_rows);
int rsed_triplets_count(const rsed_model_t* model, int64_t n_rows, const int32_t* orbit_of_row,
                        const int32_t* row_of_orbit, const double* chi, const uint64_t* stab_mask,
                        int64_t* col_off, int64_t* nnz_out, void* scratch, size_t scratch_bytes,
                        void* stream);
int rsed_triplets_fill(const rsed_model_t* model, int64_t n_rows, const int32_t* orbit_of_row,
                       const int32_t* row_of_orbit, const double* chi, const uint64_t* stab_mask,
                       const int64_t* col_off, int64_t* rows, int64_t* cols, double* vals,
                       void* stream);
/* y_v = A x_v (v < n_vec, vectors contiguous) for a complex128 CSR matrix
 * (scipy.sparse csr_matrix @ x, symmetry_resolved_ed.py:1976).  With the
 * sector block assembled from the triplets above, this is the reference's
 * operator y = H x (MatrixFreeHamiltonian.__call__, apply_hamiltonian,
 * symmetry_resolved_ed.py:1965-1976, 1979-2069). */
int rsed_csr_spmv(int64_t n_rows, const int64_t* row_ptr, const int32_t* col_idx,
                  const double* vals, int32_t n_vec, const double* x, double* y, void* stream);

/* ---- K9: sector state -> Fock amplitudes ------------------------------------
 * Replaces _expand_sector_state_to_fock_amplitudes
 * (observables/entanglement_spectrum.py:82-145).  x_orbit holds the sector
 * vector in orbit layout (complex128 per orbit, zero outside the sector), chi
 * the sector's |G| characters.  For every basis state (table rank r) amp[r] =
 * sum over g with g(s) = mask(r), ascending, of
 * x[s] / sqrt(|G| |Stab(s)|) * conj(chi(g)) * phase_g(s) (product form),
 * representatives with |x| <= atol skipped, amplitudes <= atol set to 0, then
 * the whole vector scaled to unit norm; masks[r] (optional, NULL = skip) gets
 * the state's mask.  *norm2_out receives the norm before scaling (the call
 * synchronises the stream); RSED_EINVAL if it is <= atol. */
size_t rsed_fock_scratch_bytes(int64_t n_states);
int rsed_fock_expand(const rsed_group_t* grp, const rsed_entry_t* table, int64_t n_orbits,
                     const uint64_t* repr_masks, const uint64_t* stab_mask, const double* x_orbit,
                     const double* chi, double atol, double* amp, uint64_t* masks, double* norm2_out,
                     void* scratch, size_t scratch_bytes, void* stream);

/* Overlap matrices of dense Fock-amplitude states, for the Berry links of
 * many_body_chern_number (replaces _fock_amplitude_overlap and
 * _subspace_overlap_matrix, observables/many_body_chern_number.py:141-182).
 * states: device complex128 [n_slots][n_m][n_states], each level a dense
 * rank-indexed vector as rsed_fock_expand writes it.  pairs: HOST int32
 * [n_pairs][2] slot indices (a, b), each in [0, n_slots).  out: device
 * complex128 [n_pairs][n_m][n_m], out[p][i][j] = sum_r conj(a_i[r]) b_j[r],
 * the same sum order on every run.  Asynchronous on `stream`. */
size_t rsed_fock_overlap_scratch_bytes(int64_t n_states, int32_t n_m, int32_t n_pairs);
int rsed_fock_overlaps(const double* states, int64_t n_states, int32_t n_m, int32_t n_slots,
                       const int32_t* pairs, int32_t n_pairs, double* out, void* scratch,
                       size_t scratch_bytes, void* stream);

/* Resta's periodic position operator exp(2 pi i X / L) projected between two
 * symmetry sectors, for flux_charge_pump (replaces _position_operator_matrix
 * and the manifold products P[row, col], observables/charge_pump.py:102-161,
 * :465-486).  Per orbit o (representative s = repr_masks[o]):
 *   elem(o) = (1/|G|) sum_g chi_to[g] conj(chi_from[g]) z(g(s)),
 *   z(m) = product over the occupied sites j of m, ascending, of site_phase[j],
 * |elem| <= 1e-13 dropped (the reference's form: diagonal in the orbit, no
 * stabilizer terms).  x_to / x_from: device complex128 [k][n_orbits] sector
 * vectors in orbit layout (zero outside their sectors); out: device
 * complex128 [k_to][k_from], out[i][j] = sum_o conj(x_to[i][o]) elem(o)
 * x_from[j][o], the same sum order on every run.  chi_to, chi_from (|G|) and
 * site_phase (N) are device complex128 arrays.  Asynchronous on `stream`. */
size_t rsed_position_scratch_bytes(int64_t n_orbits, int32_t k_to, int32_t k_from);
int rsed_position_overlaps(const rsed_group_t* grp, int64_t n_orbits, const uint64_t* repr_masks,
                           const double* chi_to, const double* chi_from, const double* site_phase,
                           const double* x_to, int32_t k_to, const double* x_from, int32_t k_from,
                           double* out, void* scratch, size_t scratch_bytes, void* stream);

/* ---- correlators of one sector state ---------------------------------------
 * One-body density matrix rho[i][j] = <psi| a_i^dagger a_j |psi> (replaces the
 * orbit loops of off_diagonal_long_range_order,
 * observables/off_diagonal_long_range_order.py:77-140): x_orbit is the sector
 * vector in orbit layout (complex128, zero outside the sector), member/sector
 * the sector's membership bit per orbit, chi its |G| characters; rho is
 * device complex128 [N][N] (row i, column j, 0-based sites).  A hop between
 * the two species of a two-species basis contributes zero.  Asynchronous on
 * `stream`; the sums run in a fixed order for a given device. */
size_t rsed_obdm_scratch_bytes(int32_t n_site);
int rsed_one_body_density(const rsed_group_t* grp, const rsed_entry_t* table, int64_t n_orbits,
                          const uint64_t* repr_masks, const uint64_t* stab_mask, const uint64_t* member,
                          int32_t sector, const double* chi, const double* x_orbit, double* rho,
                          void* scratch, size_t scratch_bytes, void* stream);

/* Density pairs of one sector state over the representatives (the orbit sum
 * of _build_density_correlation_matrix, observables/static_structure_factor.py:
 * 54-149, before the sum over the group): pairs[a][b] = sum_o |x_o|^2
 * n_a(s_o) n_b(s_o), device float64 [N][N].  The caller forms
 * <n_i n_j> = (1/|G|) sum_g pairs[a][b] at i = g(a), j = g(b). */
size_t rsed_density_pairs_scratch_bytes(int32_t n_site);
int rsed_density_pairs(int32_t n_site, int64_t n_orbits, const uint64_t* repr_masks, const double* x_orbit,
                       double* pairs, void* scratch, size_t scratch_bytes, void* stream);

/* ---- K8: batched thick-restart block Lanczos -------------------------------
 * Replaces diagonalize_block_matrixfree / diagonalize_block_arpack
 * (symmetry_resolved_ed.py:2214-2299, ARPACK eigs(which="SR", tol=1e-10))
 * for many sector instances at once.  State lives in caller-owned device
 * buffers described by rsed_lanczos_t.  rsed_lanczos_iterate advances every
 * active instance by n_iter block steps without host synchronisation or
 * allocation (capturable in a CUDA graph); per-instance status is read from
 * state[16*i + 1] (0 running, 1 converged, RSED_E* on failure); state[16*i + 3]
 * counts block steps + 1, state[16*i + 11] the steps that took a single
 * Gram-Schmidt pass, state[16*i + 12] the basis blocks (plus W) read by all
 * executed Gram-Schmidt passes and state[16*i + 13] those passes (each
 * pass's update reads one block more and writes one). */
typedef struct {
  int32_t n_inst;        /* instances (sector solves) in the batch */
  int32_t n_slots;       /* basis blocks before a thick restart (n_slots*bmax <= 64) */
  int32_t nev;           /* wanted lowest eigenpairs per instance */
  int32_t keep_blocks;   /* blocks kept at a restart (keep_blocks*bmax <= 16) */
  int32_t max_restarts;  /* restart cap -> RSED_ENOTCONV */
  int32_t precision;     /* matvec precision: 64 or 32 */
  int32_t bmax;          /* largest instance block size (<= 8) */
  int32_t chunk_rows;    /* rows per reduction chunk */
  int32_t pm;            /* leading dimension of the projected matrices >= (n_slots+1)*bmax */
  int32_t reserved;      /* bit 0: adaptive single Gram-Schmidt pass (pass 1 removes the part of
                          * the recurrence known from the projected matrix; pass 2 is skipped per
                          * instance when no Cholesky pivot of pass 1 lost more than 7/8 of its
                          * column's norm^2) */
  double tol;            /* converged when ||r_j|| <= tol * max(1, |theta_j|) for j < nev */
  const int32_t* inst_col0;  /* n_inst: first column of each instance */
  const int32_t* inst_b;     /* n_inst: block size of each instance */
  double* V;             /* (n_slots+2) x n_orbits x ld complex128: basis slots, last = current block */
  double* W;             /* n_orbits x ld complex128 */
  float* Xf;             /* n_orbits x ld complex64 current block (precision 32), else NULL */
  double* P;             /* n_inst x pm x pm complex128 projected matrices */
  double* coef;          /* rsed_lanczos_coef_len() doubles */
  double* partial;       /* partial_len doubles */
  int64_t partial_len;   /* >= rsed_lanczos_partial_len() */
  double* ritz_val;      /* n_inst x pm */
  double* ritz_vec;      /* n_inst x pm x pm complex128 */
  double* resid;         /* n_inst x pm */
  int32_t* state;        /* n_inst x 16 */
} rsed_lanczos_t;
int64_t rsed_lanczos_partial_len(int64_t n_orbits, int32_t chunk_rows, int32_t n_inst,
                                 int32_t n_slots);
int64_t rsed_lanczos_coef_len(int32_t n_inst, int32_t n_slots);
int rsed_lanczos_max_block(void);
int rsed_lanczos_max_keep(void);
int rsed_lanczos_max_projected(void);
/* One-time kernel attribute set-up; call before capturing a graph. */
int rsed_lanczos_prepare(void);
/* The start block is read from the columns of W; it is orthonormalised
 * (Cholesky QR twice) into basis slot 0. */
int rsed_lanczos_start(const rsed_model_t* model, const rsed_sectors_t* sec, rsed_lanczos_t* st,
                       void* stream);
int rsed_lanczos_iterate(const rsed_model_t* model, const rsed_sectors_t* sec, rsed_lanczos_t* st,
                         int32_t n_iter, int32_t check_every, int32_t apply_variant, void* stream);
/* n_iter block steps that launch the Ritz check and the restart only after
 * the last step (ritz_last != 0) or not at all.  Same state as
 * rsed_lanczos_iterate with the same n_iter when neither a restart (the
 * basis reaching n_slots + 1 blocks) nor a periodic check falls due before
 * the last step -- the active instances all advance one block per step, so
 * restarts come n_slots steps after rsed_lanczos_start and every
 * n_slots - keep_blocks steps after that.  A restart that falls due inside
 * the span stops its instance with RSED_EINVAL at the next Gram pass. */
int rsed_lanczos_iterate_span(const rsed_model_t* model, const rsed_sectors_t* sec, rsed_lanczos_t* st,
                              int32_t n_iter, int32_t ritz_last, int32_t check_every,
                              int32_t apply_variant, void* stream);
/* FP64 Rayleigh-Ritz refinement of converged instances (typically after an
 * FP32-matvec solve): the thick-restart basis (keep_blocks*b Ritz vectors
 * plus the residual block) is re-projected with the FP64 operator, the
 * Ritz pairs recomputed, and the true FP64 residual norms ||H u - theta u||
 * written to resid[inst*pm + j].  Needs n_slots >= 2*keep_blocks + 1. */
int rsed_lanczos_rayleigh_ritz(const rsed_model_t* model, const rsed_sectors_t* sec,
                               rsed_lanczos_t* st, int32_t apply_variant, void* stream);
/* The thick restart alone, as rsed_lanczos_iterate runs it after a Ritz
 * check: every instance with state[S_RESTART_NB] = nb_old > 0 gets
 * V_j = sum_{l < (nb_old-1)*b} V_l S[l][j] for j < keep_blocks*b (S =
 * ritz_vec, columns of block j/b, column j%b) and its residual block (slot
 * nb_old-1) moved to slot keep_blocks.  Instances with nb_old = 0 are left
 * alone.  No reference counterpart (the reference's ARPACK restarts inside
 * scipy); exposed so the restart can be checked on its own. */
int rsed_lanczos_restart(const rsed_model_t* model, const rsed_sectors_t* sec, rsed_lanczos_t* st,
                         void* stream);
/* The whole thick-restart loop for every active instance in ONE launch: one
 * thread-block cluster of cluster_size (1..8) CTAs per instance, each CTA
 * owning a slice of the orbit rows; Gram reductions go through distributed
 * shared memory, the projected eigenproblem is solved by the cluster's first
 * CTA.  Block sizes must divide 32.  Runs at most max_iter block steps;
 * per-instance status and the Ritz data are left in `st` as after
 * rsed_lanczos_iterate, so rsed_lanczos_rayleigh_ritz/_extract follow. */
int rsed_lanczos_persistent(const rsed_model_t* model, const rsed_sectors_t* sec, rsed_lanczos_t* st,
                            int32_t cluster_size, int32_t max_iter, void* stream);
/* Ritz vectors of the nev lowest pairs of the last check:
 * U[(inst*nev + j)*u_stride + orbit] (complex128). */
int rsed_lanczos_extract(const rsed_model_t* model, const rsed_sectors_t* sec, rsed_lanczos_t* st,
                         double* U, int64_t u_stride, void* stream);

/* Row gather / scatter between a sector's compact basis order and the
 * orbit-row layout (complex128): dst[r*dst_stride] = src[orbit_of_row[r]*src_ld + src_col]
 * and the converse. */
int rsed_gather_rows(int64_t n_rows, const int32_t* orbit_of_row, const double* src, int64_t src_ld,
                     int32_t src_col, double* dst, int64_t dst_stride, void* stream);
int rsed_scatter_rows(int64_t n_rows, const int32_t* orbit_of_row, const double* src,
                      int64_t src_stride, double* dst, int64_t dst_ld, int32_t dst_col, void* stream);
/* n_cols orbit-layout columns (column j at src + j*src_col_stride) into a
 * row-major [n_rows, dst_ld] complex128 block in one launch:
 * dst[r*dst_ld + j] = src[j*src_col_stride + orbit_of_row[r]]. */
int rsed_gather_block(int64_t n_rows, const int32_t* orbit_of_row, const double* src, int32_t n_cols,
                      int64_t src_col_stride, double* dst, int64_t dst_ld, void* stream);
/* The first n_cols columns of a row-major [n_rows, src_ld] complex128 block in
 * one launch: dst[orbit_of_row[r]*dst_ld + dst_col0 + j] = src[r*src_ld + j]. */
int rsed_scatter_block(int64_t n_rows, const int32_t* orbit_of_row, const double* src, int32_t n_cols,
                       int64_t src_ld, double* dst, int64_t dst_ld, int32_t dst_col0, void* stream);
int rsed_device_sync(void* stream);
/* Kernel launches issued by the library so far (process-wide counter; a
 * CUDA graph replay re-runs the launches counted while it was captured). */
long long rsed_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* RSED_H_ */
