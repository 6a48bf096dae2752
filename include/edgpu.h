/*
 * edgpu.h -- C ABI of the B200 sector-Lanczos engine (libedgpu.so).
 *
 * The engine replaces the hot path of EDlattice (aamaricci/ED_Lattice): the sector Fock
 * basis, the H x v product and the Lanczos tridiagonalisation behind the GF/CHI/OC
 * builders. Every entry point below names the reference interface it stands in for
 * (paths relative to the EDlattice project root).
 *
 * Conventions
 *  - Plain C types only; host pointers unless the name says _dev.
 *  - Every call returns an int status: EDG_OK (0) or a negative EDG_ERR_* code. No call
 *    aborts the process; edg_last_error() gives a one-line message for the calling thread.
 *  - Vector layout is the reference's: element i (0-based) = iup + idw*DimUp with iup the
 *    up-spin basis rank (fastest) and idw the down-spin rank (src/SECTOR.f90:443-480).
 *  - Sites and spins are 1-based where the reference's arguments are (site io, ispin).
 *  - Sizes are int64_t: sectors above 2^31 states are supported (the reference's are int32).
 *  - One sector handle is used by one host thread at a time; separate handles are
 *    independent (the reference keeps one active sector in module globals,
 *    src/DIAG/HAMILTONIAN_COMMON.f90:13-40).
 */
#ifndef EDGPU_H
#define EDGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  EDG_OK = 0,
  EDG_ERR_ARG = -1,          /* invalid argument (replaces the reference's `stop` on bad input) */
  EDG_ERR_CUDA = -2,         /* a CUDA runtime call failed */
  EDG_ERR_NOMEM = -3,        /* HBM admission refused or allocation failed */
  EDG_ERR_UNSUPPORTED = -4,  /* model feature outside the engine (e.g. complex Hij on device) */
  EDG_ERR_STATE = -5,        /* handle in the wrong state */
  EDG_ERR_NOCONV = -6,       /* eigen-solver did not converge */
  EDG_ERR_NODEVICE = -8      /* no CUDA device visible */
};

/* H x v forms: the reference's ed_sparse_H switch (src/INPUT_VARS.f90:151,
 * src/DIAG/HAMILTONIAN.f90:148-160). STORED = spMatVec over tables built once per sector;
 * DIRECT = directMatVec, matrix elements generated on the fly. */
enum { EDG_FORM_STORED = 0, EDG_FORM_DIRECT = 1 };

/* Precision of the device Lanczos vectors. Scalars (alpha, beta, dots) are always FP64. */
enum { EDG_PREC_F64 = 0, EDG_PREC_F32 = 1 };

/* Ground-state modes: plain FP64 Lanczos, or FP32 Lanczos + restarted FP64 refinement.
 * OR with EDG_GS_E0_ONLY to skip building the final eigenvector (time-to-E0 runs). */
enum { EDG_GS_F64 = 0, EDG_GS_F32_REFINE = 1, EDG_GS_E0_ONLY = 0x100 };

typedef struct edg_model_s edg_model;
typedef struct edg_sector_s edg_sector;

const char* edg_last_error(void);
int edg_device_count(int* n);
/* Hand the device memory that the library's allocation pool holds for reuse (up to a quarter
 * of the current device's memory, kept between sectors) back to the driver, after waiting for
 * the device. No counterpart in the reference. */
int edg_release_cached_memory(void);

/* ------------------------------------------------------------------ model
 * Replaces Hij_init/Hij_add_link/Hij_build/Hij_get (src/GRAPH_MATRIX.f90:79-344) plus the
 * hot-path input keys ULOC, XMU, HFMODE, ED_FILLING (src/INPUT_VARS.f90:106-166).
 * hij_re/hij_im: Hij(1,io,jo) row-major [io*ns+jo], Norb=1; hijdw_*: Hij(2,:,:) when
 * nspin==2 (NULL otherwise). hij_im/hijdw_im may be NULL (real Hij). The Hermiticity check
 * of Hij_build (tolerance 1e-6, src/GRAPH_MATRIX.f90:325) returns EDG_ERR_ARG. */
int edg_model_create(int ns, int nspin, const double* hij_re, const double* hij_im,
                     const double* hijdw_re, const double* hijdw_im, double uloc, double xmu,
                     int hfmode, int ed_filling, edg_model** out);
int edg_model_destroy(edg_model* m);

/* ------------------------------------------------------------------ sector numbering
 * get_Sector / get_Nup / get_Ndw (src/SECTOR.f90:370-424) and binomial
 * (src/SETUP.f90:336-358). */
int edg_get_sector(int ns, int nup, int ndw);
int edg_get_nup(int ns, int isector);
int edg_get_ndw(int ns, int isector);
int64_t edg_binomial(int n, int k);

/* ------------------------------------------------------------------ sector lifecycle
 * build_Hv_sector(isector) / delete_Hv_sector() / vecDim_Hv_sector(isector)
 * (src/DIAG/HAMILTONIAN.f90:53-239) with build_sector (src/SECTOR.f90:69-115) done on the
 * device: Gosper enumeration of the Nup/Ndw bitstrings, combinatorial-rank index maps and,
 * for EDG_FORM_STORED, the per-spin hop tables of ed_buildh
 * (src/DIAG/HAMILTONIAN_STORED_HxV.f90:21-126). */
int edg_sector_create(const edg_model* m, int nup, int ndw, int form, edg_sector** out);
int edg_sector_destroy(edg_sector* s);
int edg_sector_dims(const edg_sector* s, int64_t* dim, int64_t* dimup, int64_t* dimdw);
/* Reals per vector of this sector: dim, or 2*dim when the model's Hij is complex. The
 * reference's vectors are complex(8) throughout; with complex Hij every vector argument of
 * this API (host or device: start vectors, H x v operands, states) holds dim complex
 * elements interleaved (re, im), device ones 2*sizeof(T)-aligned, and the Lanczos scalars
 * stay real. edg_sector_dense(_dev) then writes dim x dim complex entries. */
int edg_sector_vlen(const edg_sector* s, int64_t* vlen);
/* Copy the device-built maps Hsector%H(1)%map / H(2)%map (bitstrings, ascending). */
int edg_sector_get_maps(const edg_sector* s, int32_t* map_up, int32_t* map_dw);
/* Copy one spin's hop table (spin 1 = spH0ups(1), 2 = spH0dws(1)) as CSR over target rows:
 * rowptr[dim+1], cols[nnz] (source ranks, ascending per row), vals[nnz] (real part). Pass
 * NULL arrays to get *nnz only. */
int edg_sector_get_hops(const edg_sector* s, int spin, int64_t* rowptr, int32_t* cols,
                        double* vals, int64_t* nnz);
/* Hand back the sector's work buffers (Lanczos vectors, the FP32 ground-state basis, block
 * chain vectors) to the library's pool, keeping its tables and its state buffer: between a
 * ground state and the response chains of a sector whose vectors take tens of GB. Later
 * calls allocate again on demand. No counterpart in the reference. */
int edg_sector_release_work(edg_sector* s);
/* Run this sector's work on a caller-owned stream (cudaStream_t passed as void*). */
int edg_sector_set_stream(edg_sector* s, void* stream);

/* ------------------------------------------------------------------ H x v
 * dd_sparse_HxV(Nloc,v,Hv) (src/VARS_GLOBAL.f90:102-108), the callback that
 * spHtimesV_p points to (spMatVec / directMatVec). Host complex(8) vectors, interleaved
 * (re,im); Hv is overwritten. With real Hij, H acts on the real and the imaginary parts
 * separately; with complex Hij the complex H is applied, the stored form with the
 * conjugated hop values the reference stores (src/DIAG/stored/H_up.f90:19-21) and the
 * direct form with Hij itself (src/DIAG/direct/HxV_up.f90:24). nloc must equal the sector
 * dimension (the reference stops with "Nloc != dim(isector)",
 * src/DIAG/HAMILTONIAN_DIRECT_HxV.f90:33). */
int edg_hxv_z(edg_sector* s, int64_t nloc, const double* v, double* hv);
/* Same on real host vectors (real Hij only). */
int edg_hxv_d(edg_sector* s, int64_t nloc, const double* v, double* hv);
/* Autotuner of the stored-form H x v (real Hij): times each candidate pair of down-spin and
 * up-spin pass kernels (4 x 4 for FP32 vectors, 4 x 1 for FP64) on `reps` applications to
 * scratch vectors of this sector (after one untimed application each), with CUDA events on
 * the sector's stream, and keeps the fastest pair for that precision: the H x v, the fused
 * Lanczos steps and the block chains of this sector then use it. Candidate k = nup*down + up
 * (nup = 4 for FP32, 1 for FP64): down 0 hop-balanced row groups, 1 block-staged rows (one
 * CTA per SM), 2 block-staged rows (two CTAs per SM), 3 the single-pass H x v (the whole
 * product in one launch, for vectors that sit in L2; the up choice is then unused); up (FP32)
 * 0 32-bit SELL schedule,
 * 1 packed 16-bit schedule with negated copies, 2 packed 16-bit schedule with sign bits,
 * 3 Kronecker schedule (hops inside the low or the high half of the sites from per-half
 * tables, the rest from a per-column table). ms (may be NULL) receives each candidate's ms
 * per H x v, *ncand their number, *best the index kept. FP64 results are the same bits for
 * every pair; the FP32 packed and Kronecker up passes change the order of a row's terms.
 * Untuned real stored sectors of at most 500,000 states use the single pass (candidate 12
 * for FP32, 3 for FP64), other sectors candidate 0. No counterpart in the reference. */
int edg_sector_autotune(edg_sector* s, int precision, int reps, double* ms, int* ncand, int* best);
/* Pin the H x v kernel pair of this sector for one precision to candidate k of
 * edg_sector_autotune's list (0..15 for FP32, 0..3 for FP64). The tables of the non-default
 * kernels are built on the first call that needs them (this one, or edg_sector_autotune);
 * sectors that keep candidate 0 never build them. No counterpart in the reference. */
int edg_sector_set_kernels(edg_sector* s, int precision, int candidate);
/* Device-resident forms (vectors in HBM, reference layout); stream-ordered, no sync. */
int edg_hxv_dev_f64(edg_sector* s, const double* dv, double* dhv);
int edg_hxv_dev_f32(edg_sector* s, const float* dv, float* dhv);
/* Slab forms of the stored H x v for a sector whose vectors are split over the ranks of a
 * process group by rows (the down-spin index idw of element iup + idw*DimUp); the sector
 * object itself holds only the O(DimUp + DimDw) tables. Replaces, for sectors beyond one
 * GPU's memory, the reference's MPI split of spMatVec (src/DIAG/HAMILTONIAN_STORED_HxV.f90,
 * MPI branch), which this build does not otherwise reproduce.
 *  - cols: dv/dhv hold ALL DimDw rows of columns [col0, col0+ncols), row-major with row
 *    length ncols (the transpose of the row slabs); dhv = (diag + H_dw x I) dv there.
 *  - rows: dv/dhv hold rows [row0, row0+nrows), row length DimUp; dhv += (I x H_up) dv.
 * The column form, then the row form on its transposed result, is edg_hxv_dev_* bit for bit.
 * Real stored-form sectors; stream-ordered, no sync. No counterpart in the reference. */
int edg_hxv_cols_dev_f64(edg_sector* s, int64_t col0, int64_t ncols, const double* dv, double* dhv);
int edg_hxv_cols_dev_f32(edg_sector* s, int64_t col0, int64_t ncols, const float* dv, float* dhv);
int edg_hxv_rows_dev_f64(edg_sector* s, int64_t row0, int64_t nrows, const double* dv, double* dhv);
int edg_hxv_rows_dev_f32(edg_sector* s, int64_t row0, int64_t nrows, const float* dv, float* dhv);

/* ------------------------------------------------------------------ Lanczos
 * tridiag_Hv_sector(isector,vvinit,alanc,blanc,norm2) (src/DIAG/HAMILTONIAN.f90:242-275)
 * with the recurrence of sp_lanc_tridiag: norm2=<v|v>, v/=sqrt(norm2), then nlanc steps;
 * alanc[j]=a_{j+1}, blanc[0]=0, blanc[j]=b_{j+1} (the reference's blanc(1) unused
 * convention, src/GF/GF_ELECTRONS.f90:445-447). Stops early when b < threshold; the rest
 * stays zero; *nsteps = steps taken. vvinit is a host real vector of the sector dimension.
 * precision: EDG_PREC_F64 or EDG_PREC_F32 (FP32 vectors, FP64 scalars). */
int edg_tridiag_d(edg_sector* s, const double* vvinit, int nlanc, double threshold, int precision,
                  double* alanc, double* blanc, double* norm2, int* nsteps);
/* Same from a device vector (not modified). */
int edg_tridiag_dev_f64(edg_sector* s, const double* dvinit, int nlanc, double threshold,
                        int precision, double* alanc, double* blanc, double* norm2, int* nsteps);

/* Allocation-free variant of edg_tridiag_dev_f64 (FP64 only). It has no counterpart in the
 * reference: it exists for callers that cannot allocate device memory themselves, such as a
 * host code whose device memory is owned by another runtime's pool or arena, or a loop that
 * must never wait on the allocator. All scratch (three Lanczos vectors, reduction partials,
 * scalar slots) lives in one file-scope device array of about 25 MB that every GPU loading
 * the library holds until exit; the call allocates nothing. Limits: vector length (the
 * sector dimension, 2*dim for a complex sector) <= 2^20 and nlanc <= 1024, else
 * EDG_ERR_ARG; a complex start vector must be 16-byte aligned. Calls share that array (it keeps the previous
 * call's contents; the call clears what must start at zero), so calls that overlap on the
 * GPU race and must be serialised by the caller. The first call on a device looks up the
 * array's address (cudaGetSymbolAddress) and should come before any stream capture. */
int edg_tridiag_dev_f64_noalloc(edg_sector* s, const double* dvinit, int nlanc, double threshold,
                                double* alanc, double* blanc, double* norm2, int* nsteps);

/* Ground state: the contract of sp_lanc_eigh(Hv_p,E,v,Nitermax,threshold) as called from
 * ed_diag_d (src/DIAG/DIAG.f90:212-217). v0: host start vector or NULL for the seeded
 * uniform[-1,1) start vector of edg_random_vector. Stops when the a-posteriori error of the
 * lowest Ritz value, (b_{m+1} |z_m|)^2 / gap, falls below 0.1*tol*|E0| (fallbacks: E0
 * moves by less than 0.01*tol*|E0| in a step, b underflows, or maxit). mode: EDG_GS_F64
 * or EDG_GS_F32_REFINE (FP32 phase to max(tol, 2e-7), then FP64 from its Ritz vector).
 * evec (host, may be NULL) receives the normalised eigenvector. *niter = total H x v
 * applications. */
int edg_ground_state(edg_sector* s, const double* v0, uint64_t seed, int maxit, double tol, int mode,
                     double* e0, double* evec, int* niter);
/* Device variant: the eigenvector stays on the device in the sector's state buffer; copy
 * with edg_state_get or use in the excitation builders below. */
int edg_ground_state_keep(edg_sector* s, const double* v0, uint64_t seed, int maxit, double tol,
                          int mode, double* e0, int* niter);
/* H x v applications of the last ground-state run, split by vector precision (FP32 phase,
 * FP64 phase). No counterpart in the reference (sp_lanc_eigh reports no statistics). */
int edg_ground_state_stats(const edg_sector* s, int* n_f32, int* n_f64);
/* Lowest k (1..16) eigenpairs of a sector: the sp_eigh (ARPACK) branch of ed_diag_d,
 * Neigen = min(dim, lanc_nstates_sector) states per sector for the finite-temperature state
 * list (src/DIAG/DIAG.f90:144-146,191-202). FP64 Lanczos with full reorthogonalisation
 * (classical Gram-Schmidt with its second pass from the Gram matrix of the basis). Real
 * sectors: thick-restarted, the exact-shift form of ARPACK's implicit restart, with the
 * reference's basis size Ncv = 10 k (at least 2k + 16; fewer if HBM is short): when the
 * basis is full its k + (Ncv - k)/4 lowest Ritz vectors and the residual direction start the
 * next cycle (sectors of at most 4 Ncv states keep their whole basis), and max(maxit, 8 Ncv)
 * bounds the H x v applications. Complex sectors: one unrestarted run
 * (Gram-Schmidt applied twice) with a basis of at most min(maxit, 1024) vectors. Stops when
 * every one of the k lowest Ritz pairs has residual b |z_{m,i}| <= tol*max(1,|theta_i|), or
 * the Krylov space becomes invariant, or maxit is reached. evals[k] ascending (NaN beyond
 * dim); evecs (host, may be NULL): k normalised vectors, vector r at evecs + r*dim; resid
 * (may be NULL): the k residual estimates at exit (the caller checks them against tol);
 * *niter = H x v applications. v0 and seed as in edg_ground_state. One vector per
 * eigenspace: exactly degenerate levels inside a sector appear once (use
 * edg_sector_dense for small sectors with symmetries). */
int edg_lowest_k(edg_sector* s, int k, const double* v0, uint64_t seed, int maxit, double tol,
                 double* evals, double* evecs, double* resid, int* niter);
/* Lowest-k modes: FP64 throughout (edg_lowest_k), or FP32 bulk + FP64 refinement: the same
 * solver with FP32 basis and H x v (FP64 scalars and sums) to Ritz residuals of 1e-6, whose k
 * Ritz vectors, summed, start the FP64 solve to tol. Real Hij only (complex sectors run FP64). */
enum { EDG_LK_F64 = 0, EDG_LK_F32_REFINE = 1 };
/* edg_lowest_k with a mode; *niter counts the H x v applications of both phases. The outputs
 * are those of the FP64 phase (evals, vectors and residuals to tol). */
int edg_lowest_k_mode(edg_sector* s, int k, const double* v0, uint64_t seed, int maxit, double tol,
                      int mode, double* evals, double* evecs, double* resid, int* niter);
/* Dense sector Hamiltonian, column-major dim x dim (the matrix ed_buildh(Hmat) assembles for
 * the LAPACK branch of ed_diag_d, src/DIAG/HAMILTONIAN_STORED_HxV.f90:81-117 and
 * src/DIAG/DIAG.f90:229-235): diag + kron(H_dw, 1) + kron(1, H_up). Stored form only;
 * dim <= 16384. h: host array of dim*dim doubles; the _dev variant writes device memory
 * on the sector's stream without synchronising. */
int edg_sector_dense(edg_sector* s, double* h);
int edg_sector_dense_dev(edg_sector* s, double* dh);
int edg_state_get(const edg_sector* s, double* evec);
int edg_state_set(edg_sector* s, const double* evec);

/* Seeded start vector used by the engine and the tests: splitmix64 counter stream,
 * x_i = ((splitmix64(seed + i) >> 11) * 2^-53) * 2 - 1. */
int edg_random_vector(uint64_t seed, int64_t n, double* out);

/* ------------------------------------------------------------------ excitations
 * apply_op_CDG / apply_op_C over a whole vector, as in lanc_build_gf_electrons_diag
 * (src/GF/GF_ELECTRONS.f90:241-245,267-271; src/SECTOR.f90:217-268): out = coef*op|in>
 * (overwrite) or out += coef*op|in> (accumulate=1, the (c_i + c_j) vectors of _mix,
 * :343-353). op=+1 creates, -1 annihilates; site, spin 1-based. from/to must be the
 * sectors (Nup,Ndw) and (Nup+op,Ndw) or (Nup,Ndw+op). Device FP64 vectors. */
int edg_apply_cop_dev_f64(const edg_sector* from, const edg_sector* to, int op, int site, int spin,
                          double coef, int accumulate, const double* din, double* dout);
/* S^z_i / n_i (apply_op_Sz / apply_op_N, src/SECTOR.f90:271-341): kind 0 = Sz, 1 = N;
 * site2 > 0 adds the second site (lanc_build_spinChi_mix, src/CHI/CHI_SPIN_ELECTRONS.f90:275-279).
 * Momentum form: when qcos != NULL, out = sum_i qcos[i]*O_i|in> (real combination). */
int edg_apply_diagop_dev_f64(const edg_sector* s, int kind, int site, int site2, const double* qcos,
                             const double* din, double* dout);
/* J|psi> (lanc_ed_build_oc, src/OC/OC_ELECTRONS.f90:139-205): returns the real vector r with
 * J|psi> = i*r (real Hij). */
int edg_apply_current_dev_f64(const edg_sector* s, const double* din, double* dout);

/* Static observables of one state (lanc_observables, src/OBSERVABLES.f90:127-152): per-site
 * dens, dens_up, dens_dw, docc, magz of the device state buffer, each scaled by weight. */
int edg_observables(const edg_sector* s, double weight, double* dens, double* dens_up,
                    double* dens_dw, double* docc, double* magz);

/* Energies of the state buffer: the Norb=1 terms of lanc_energy (src/ENERGY.f90:118-226).
 * ekin = <psi|hopping|psi> (off-diagonal Hij of both spins), eknot = sum_i Hij(i,i) <n_i>
 * per spin, epot = U sum_i <n_i,up n_i,dw> + ehartree, ehartree = -U/2 sum_i <n_i> when
 * HFMODE (else 0; ENERGY.f90:343 folds it into ed_Epot the same way). Each is scaled by
 * weight and ADDED to its output (NULL outputs are skipped), as edg_observables does, so a
 * caller sums Boltzmann-weighted states. One FP64 H x v of the state. The OC Drude weight
 * (src/OC/OC_FUNCTIONS.f90:65) takes ekin from here. */
int edg_energy(edg_sector* s, double weight, double* ekin, double* epot, double* eknot,
               double* ehartree);

/* ------------------------------------------------------------------ response functions
 * One Lanczos chain per excitation, as built by the GF/CHI/OC builders:
 *  edg_gf_chain: c^+ (op=+1) or c (op=-1) on the state buffer of `from`, tridiagonalised in
 *  `to`; poles = isign*(theta_j - ei), weights = norm2*Z(1,j)^2 (add_to_lanczos_gf_normal,
 *  src/GF/GF_ELECTRONS.f90:417-457). site2 > 0 forms (c_site + c_site2).
 *  poles/weights have room for nlanc entries; *nout = entries written. */
int edg_gf_chain(const edg_sector* from, edg_sector* to, int op, int site, int site2, int spin,
                 int nlanc, int precision, double ei, double* poles, double* weights, double* norm2,
                 int* nout);
/* Spin/charge susceptibility chain (add_to_lanczos_spinChi,
 * src/CHI/CHI_SPIN_ELECTRONS.f90:305-366): vector O|psi> with O from edg_apply_diagop_dev_f64,
 * poles theta_j - ei, weights norm2*Z(1,j)^2. */
int edg_chi_chain(edg_sector* s, int kind, int site, int site2, const double* qcos, int nlanc,
                  int precision, double ei, double* poles, double* weights, double* norm2, int* nout);
/* Optical-conductivity chain (add_to_lanczos_oc, src/OC/OC_ELECTRONS.f90:223-263). */
int edg_oc_chain(edg_sector* s, int nlanc, int precision, double ei, double* poles,
                 double* weights, double* norm2, int* nout);

/* Pole sums on a frequency grid, the loop of lanc_eval_gf_electrons
 * (src/GF/GF_ELECTRONS.f90:503-508): out(z_m) += sum_k weights[k] / (z_m - poles[k]) with
 * z_m = z_re[m] + i z_im[m] (i w_n on the Matsubara axis, w + i eps on the real axis). Host
 * arrays, evaluated on the current device in FP64 with a fixed summation order. The caller
 * folds the Boltzmann factors into the weights and concatenates every state and channel of
 * one Green's function entry into one call. */
int edg_eval_poles(int64_t npoles, const double* poles, const double* weights, int64_t nz,
                   const double* z_re, const double* z_im, double* out_re, double* out_im);

/* Batched chains: k start vectors of one sector in one call, each tridiagonalised as by
 * edg_tridiag_dev_f64 (one alpha/beta sequence per column, equal bit for bit to a single
 * chain's). The k chains run in lockstep as one block: every pass (the H x V and the fused
 * recurrence) is one launch over all columns still running, a column stops at its first
 * b < threshold, and k is split into blocks whose 3k work vectors fit in free HBM. Sectors
 * without the fused stored-form passes (direct form, complex Hij, rows beyond shared memory)
 * run the chains one after another. Replaces the per-chain calls of tridiag_Hv_sector in the
 * GF/CHI builders (src/GF/GF_ELECTRONS.f90:202-290, src/CHI/CHI_SPIN_ELECTRONS.f90:189-233).
 * dvinit: k device vectors, column c at dvinit + c*vlen. alanc/blanc: [k][nlanc] row-major;
 * norm2[k]; nsteps[k]. */
int edg_tridiag_block_dev(edg_sector* s, int k, const double* dvinit, int nlanc, double threshold,
                          int precision, double* alanc, double* blanc, double* norm2, int* nsteps);
/* k Green's-function chains of one state into one target sector as a block: for chain c the
 * excitation c^+_{sites[c]} (op=+1) or c_{sites[c]} (op=-1) of spin `spin` on the state
 * buffer of `from`, plus the same operator on sites2[c] when sites2 != NULL and
 * sites2[c] > 0 (the (c_i + c_j) vectors of lanc_build_gf_electrons_mix,
 * src/GF/GF_ELECTRONS.f90:343-353); then edg_tridiag_block_dev (threshold 1e-9) and the
 * poles op*(theta_j - ei) and weights norm2*Z(1,j)^2 of add_to_lanczos_gf_normal
 * (src/GF/GF_ELECTRONS.f90:417-457), the tridiagonal eigenproblems solved on the device (one
 * implicit-QL thread per chain). poles/weights: [k][nlanc]; nout[k] entries valid per chain. */
int edg_gf_chain_block(const edg_sector* from, edg_sector* to, int op, int k, const int* sites,
                       const int* sites2, int spin, int nlanc, int precision, double ei, double* poles,
                       double* weights, double* norm2, int* nout);
/* k susceptibility chains of the state buffer of s as a block (add_to_lanczos_spinChi,
 * src/CHI/CHI_SPIN_ELECTRONS.f90:305-366): operator of chain c = kind (0 Sz, 1 N) on
 * sites[c] (+ sites2[c]), or, when qcos != NULL, the momentum combination with site weights
 * qcos[c*ns .. c*ns+ns) (sites ignored). Poles theta_j - ei, weights norm2*Z(1,j)^2, as
 * edg_gf_chain_block. */
int edg_chi_chain_block(edg_sector* s, int kind, int k, const int* sites, const int* sites2,
                        const double* qcos, int nlanc, int precision, double ei, double* poles,
                        double* weights, double* norm2, int* nout);
/* Poles and weights of k chains from their coefficients ([k][nlanc] host arrays in the
 * blanc(1)-unused convention, nsteps[k] valid steps each): the eigenproblems of
 * add_to_lanczos_gf_normal solved on the current device, one implicit-QL thread per chain
 * (src/GF/GF_ELECTRONS.f90:445-456); poles isign*(theta_j - ei), weights norm2[c]*Z(1,j)^2. */
int edg_poles_weights_block(int k, int nlanc, const double* alanc, const double* blanc,
                            const double* norm2, const int* nsteps, double ei, int isign,
                            double* poles, double* weights);

/* Tridiagonal eigenproblem (SF_LINALG eigh(diag,subdiag,Ev) as used at
 * src/GF/GF_ELECTRONS.f90:447): FP64 implicit QL, eigenvalues ascending; z1 receives the
 * first component of each eigenvector (may be NULL). d[n], e[n] with e[0] ignored. */
int edg_tridiag_eigh(int n, const double* d, const double* e, double* w, double* z1);
/* The k lowest eigenvalues of the same tridiagonal, ascending, and the magnitude of the last
 * component of each unit eigenvector (zn, may be NULL): Sturm bisection and a twisted
 * factorisation, O(k n). Stands in for the Ritz-residual test |b z_n| of ARPACK's dsaupd
 * reverse-communication loop (sp_eigh at src/DIAG/DIAG.f90:191-202); edg_lowest_k uses it
 * between steps and confirms with the QL eigenvectors before it stops. */
int edg_tridiag_lowest(int n, const double* d, const double* e, int k, double* w, double* zn);
/* poles/weights from (a,b,norm2): the loop of add_to_lanczos_gf_normal (:451-456). */
int edg_poles_weights(int n, const double* alanc, const double* blanc, double norm2, double ei,
                      int isign, double* poles, double* weights);

#ifdef __cplusplus
}
#endif

#endif /* EDGPU_H */
