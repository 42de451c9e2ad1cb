/* ipg.h — C ABI of libipg.so, the B200 (sm_100a) force-field evaluation library.
 *
 * Every entry point is extern "C", takes plain pointers and sizes, returns an int status
 * (IPG_OK = 0, negative = error) and never aborts.  Details of the last error of a
 * context are available from ipg_last_error().
 *
 * Each declaration names the reference (cesmix-mit/InteratomicPotentials.jl v0.3.2)
 * interface it replaces, as file:line within that project.
 *
 * Conventions
 *  - Positions and forces are AoS: x0 y0 z0 x1 y1 z1 ... (Julia Vector{SVector{3,Float64}}
 *    reinterpreted as a flat Float64 array).
 *  - L[3] is the orthorhombic box diagonal; INFINITY marks an open (non-periodic) axis,
 *    as in src/nnlist.jl:29 and src/BasisSystems/SNAP/utilities/utl.jl:64.
 *  - Species are 0-based int32 ids.  For pair terms they index the 64-bit species mask;
 *    for SNAP they index snap.species.
 *  - Units: the pair API takes atomic units (bohr, hartree), like the reference
 *    internals after austrip; the SNAP API takes the caller's length unit, like the
 *    reference's ustrip.
 *  - Host-pointer entry points copy inputs to the device and results back before they
 *    return.  *_dev entry points take device pointers and run on the context's stream
 *    (set with ipg_set_stream); they synchronise that stream before returning.  Inside a
 *    call the library may fork work onto a second, internal stream of the context (event
 *    fork and join, also valid inside a graph capture); it is joined before the call returns.
 *  - Ownership: the caller owns every buffer it passes.  The library owns the device
 *    scratch inside a context and grows it on demand.
 *  - Threading: one context per host thread; calls on distinct contexts are independent.
 */
#ifndef IPG_H
#define IPG_H

#include <stdint.h>

#if defined(IPG_BUILD) && defined(__GNUC__)
#define IPG_API __attribute__((visibility("default")))
#else
#define IPG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------ */
#define IPG_OK 0
#define IPG_ERR_ARG (-1)          /* invalid argument (null pointer, bad size or flag)   */
#define IPG_ERR_CUDA (-2)         /* CUDA runtime error                                  */
#define IPG_ERR_NOMEM (-3)        /* device allocation failed                            */
#define IPG_ERR_CAPACITY (-4)     /* a device-side capacity was exceeded                 */
                                  /* (-5 is not used: no kernel waits on another)         */
#define IPG_ERR_NONFINITE (-6)    /* NaN or Inf in positions                             */
#define IPG_ERR_SPECIES (-7)      /* species id out of range                             */
#define IPG_ERR_UNSUPPORTED (-8)  /* valid in the reference but not built here           */
#define IPG_ERR_NODEVICE (-9)     /* no CUDA device (or not an sm_100 device)            */

/* ---- opaque handles ------------------------------------------------------------------ */
typedef struct ipg_ctx ipg_ctx;
typedef struct ipg_nlist ipg_nlist;
typedef struct ipg_snap ipg_snap;

/* ---- context ------------------------------------------------------------------------- */
/* Creates a context on CUDA device `device` with its own non-blocking stream. */
IPG_API int ipg_create(int device, ipg_ctx** out);
IPG_API int ipg_destroy(ipg_ctx* ctx);
/* Message of the last error on ctx ("" if none).  Valid until the next call on ctx. */
IPG_API const char* ipg_last_error(const ipg_ctx* ctx);
/* Runs subsequent *_dev calls on `stream` (a cudaStream_t, or NULL for the context's own). */
IPG_API int ipg_set_stream(ipg_ctx* ctx, void* stream);
/* Library version as MAJOR*10000 + MINOR*100 + PATCH. */
IPG_API int ipg_version(void);
/* Number of kernels this context has launched so far (for launch accounting).
 * Instrumentation with no counterpart in the reference. */
IPG_API int ipg_launch_count(const ipg_ctx* ctx, int64_t* out);
/* Per-kernel device timing (instrumentation with no counterpart in the reference):
 * when enabled, the dominant kernels are bracketed by CUDA events on the context's
 * stream.  ipg_timing_read returns the summed milliseconds and launch count recorded
 * under `kernel` since the last read, and resets them.  Names: "neighbor" (the whole
 * neighbor build), "pair_eval" (pair potentials), and the SNAP kernels "snap_utot" (Utot),
 * "snap_atom" (the Y kernel of the adjoint path, or the per-atom block kernel),
 * "snap_pair" (per-neighbor adjoint forces), "snap_gather" (force gather), "snap_zrows" (Z),
 * "snap_bdesc" (B), "snap_dbfused" (plain dB/dr), "snap_contract" (plain-path contraction),
 * "snap_vsum" and "snap_gbeta" (beta pullback; "snap_vsum" also carries the Utot tangent of
 * the position pullback), "snap_hvp_y" (its two polarized Y evaluations), "snap_hvp" (the
 * rest of the exact Hessian-vector product: the pair part, or the per-atom forward-mode
 * kernel).  Unknown names read as zero. */
IPG_API int ipg_timing_enable(ipg_ctx* ctx, int on);
IPG_API int ipg_timing_read(ipg_ctx* ctx, const char* kernel, double* total_ms, int64_t* launches);

/* ---- neighbor lists -------------------------------------------------------------------
 * Replaces neighborlist(s, rcut) (src/nnlist.jl:23-46) and neighborlist(A, snap)
 * (src/BasisSystems/SNAP/utilities/utl.jl:38-101).
 *
 * mode IPG_NLIST_HALF: pairs (i, j > i) whose Distances.PeriodicEuclidean distance is
 *   <= cut[0]; r = x_i - x_j under minimum image (get_displacement, src/nnlist.jl:18-21).
 * mode IPG_NLIST_FULL: pairs (i, j != i) with |r|^2 <= cut[s_i * nspecies + s_j] and
 *   r = x_j - x_i (utl.jl:87-89); the candidate radius is sqrt(max cut) — or, with
 *   IPG_NLIST_LITERAL_SQRT, the reference's literal sqrt(sqrt(max cut)) (utl.jl:81).
 * Within each atom the neighbors are sorted by index (inrange(..., true), utl.jl:81). */
#define IPG_NLIST_HALF 0
#define IPG_NLIST_FULL 1
#define IPG_NLIST_LITERAL_SQRT 0x100
IPG_API int ipg_neighbor_build(ipg_ctx* ctx, int64_t n, const double* pos, const double L[3], const int32_t* species,
                       int32_t nspecies, const double* cut, int32_t mode, ipg_nlist** out);
IPG_API int ipg_nlist_size(const ipg_nlist* nl, int64_t* npairs);
/* The pair count of the list ipg_neighbor_build would return, without building or copying
 * it (cell list and one counting walk on the device). */
IPG_API int ipg_neighbor_count(ipg_ctx* ctx, int64_t n, const double* pos, const double L[3], const int32_t* species,
                       int32_t nspecies, const double* cut, int32_t mode, int64_t* npairs);
/* offsets [n+1], j [npairs] (0-based), r [3*npairs]; any may be NULL. */
IPG_API int ipg_nlist_export(const ipg_nlist* nl, int64_t* offsets, int32_t* j, double* r);
IPG_API int ipg_nlist_free(ipg_nlist* nl);

/* ---- empirical pair potentials ---------------------------------------------------------
 * One ipg_pair_term is one EmpiricalPotential; a list of terms with coefficients is a
 * LinearCombinationPotential (src/mixed/linear_combination_potential.jl:7-39).  Each
 * term keeps its own cutoff and species filter (src/types/empirical_potential.jl:26-43:
 * a pair counts when BOTH species are in the term's set).
 * params by kind (all atomic units):
 *   IPG_PAIR_LJ      eps, sigma                   src/empirical/lj.jl:35-36
 *   IPG_PAIR_BM      A, rho, sigma, C, D          src/empirical/bm.jl:38-39
 *   IPG_PAIR_COUL    q1, q2                       src/empirical/coulomb.jl:36-37
 *   IPG_PAIR_MORSE   D, alpha, sigma              src/empirical/morse.jl:36-39
 *   IPG_PAIR_ZBL     Z1, Z2, e                    src/empirical/zbl.jl:27-36
 *   IPG_PAIR_MOCK_R2 seed  (E = seed R^2, f = seed R^2 r; test/mocks.jl:22-34)            */
#define IPG_PAIR_LJ 1
#define IPG_PAIR_BM 2
#define IPG_PAIR_COUL 3
#define IPG_PAIR_MORSE 4
#define IPG_PAIR_ZBL 5
#define IPG_PAIR_MOCK_R2 6
#define IPG_MAX_PAIR_TERMS 16
typedef struct ipg_pair_term {
  int32_t kind;
  int32_t reserved;
  double coeff;          /* linear-combination coefficient                           */
  double rcut;           /* get_rcutoff(p)                                           */
  uint64_t species_mask; /* bit s set <=> species s in get_species(p); ~0 = missing  */
  double params[8];
} ipg_pair_term;

/* What to compute (bit flags). */
#define IPG_WANT_E 1u
#define IPG_WANT_F 2u
#define IPG_WANT_W 4u
/* ipg_pair_eval_dev only: replay a CUDA graph of the whole evaluation (cell list, pair
 * tiles, gather, reductions).  The first call with a given (n, L, terms, device buffers,
 * flags) runs eagerly and captures the graph; later calls with the same key upload the cell
 * grid and launch the graph once (an MD loop's step with fixed buffers).  Open boxes
 * (L = inf) and failed captures run eagerly.  Results are those of the eager call. */
#define IPG_PAIR_GRAPH 8u

/* energy_and_force / potential_energy / force / virial_stress for an EmpiricalPotential
 * or a LinearCombinationPotential (empirical_potential.jl:49-77,
 * linear_combination_potential.jl:27-39).  E [1], F [3n], W6 [6] = [xx,yy,zz,zy,zx,yx]
 * (empirical_potential.jl:63-64); outputs not selected by `flags` may be NULL. */
IPG_API int ipg_pair_eval(ipg_ctx* ctx, int64_t n, const double* pos, const int32_t* species, const double L[3],
                  const ipg_pair_term* terms, int32_t nterms, double* E, double* F, double* W6, uint32_t flags);
IPG_API int ipg_pair_eval_dev(ipg_ctx* ctx, int64_t n, const double* d_pos, const int32_t* d_species, const double L[3],
                      const ipg_pair_term* terms, int32_t nterms, double* d_E, double* d_F, double* d_W6,
                      uint32_t flags);
/* ipg_pair_eval_dev for callers that cannot allocate device memory (no counterpart in
 * the reference): an MD engine that owns all device memory up front, or a host that
 * holds only a stream and device buffers and must not create a context (creating one
 * allocates).  Same inputs, outputs and results; no context, no allocation.  Its scratch
 * is a fixed device array of about 4.3 MB that every GPU loading the library keeps until
 * exit; at most 65,536 atoms (larger n returns IPG_ERR_CAPACITY before any launch).
 * Work is enqueued on `stream` (a cudaStream_t, NULL = legacy default stream) on the
 * current device and not synchronised.  Calls share the scratch array: calls that overlap
 * on the GPU race, so serialise them (one stream).  The first call on a device resolves
 * the scratch address; make it before any stream capture.  That address belongs to the
 * device's CUDA context at the first call and is kept until exit: do not call this entry
 * point on a device after cudaDeviceReset there.  Device-side input errors are not reported
 * (there is no status word to read without a synchronisation): a non-finite position is
 * placed in an arbitrary cell and gives non-finite results, and a species id outside 0..63
 * is clamped into that range. */
IPG_API int ipg_pair_eval_noalloc(void* stream, int64_t n, const double* d_pos, const int32_t* d_species,
                                  const double L[3], const ipg_pair_term* terms, int32_t nterms, double* d_E,
                                  double* d_F, double* d_W6, uint32_t flags);

/* ---- SNAP -------------------------------------------------------------------------------
 * ipg_snap_params mirrors SNAP{S,T} (src/BasisSystems/SNAP/types/types.jl:8-25).
 * chem_flag (explicit multi-element SNAP; it must equal bnorm_flag, snap.jl:10-13): one Utot
 *   per element (the neighbor's element, compute_ui.jl:155-175), Z per ordered element pair
 *   (compute_z.jl:5-61), B and dB/dr per element triple (compute_b.jl:15-95, 104-342), so
 *   K = idxb_max * nspecies^3 (utl.jl:8-25).  The Z index of compute_z.jl:44-47 writes every
 *   pair into the first block; literal_chem_z reproduces that, the default keeps one block per
 *   pair.  bzero shifts the centre element's triple (every triple with wselfall_flag).
 * quadratic_flag (quadratic SNAP, the option of LAMMPS_SNAP/snap.jl:45-47): the K linear
 *   components are followed by 0.5 B_k^2 and B_k B_l (l > k), K + K(K+1)/2 in all; beta and
 *   the descriptors use that length.
 * With chem_flag or quadratic_flag the evaluation runs the per-atom element-resolved kernel
 *   (forces through dB/dr in either mode) and ipg_snap_vjp's position pullback returns
 *   IPG_ERR_UNSUPPORTED.  wselfall_flag puts wself on every element's Utot.                */
#define IPG_MAX_SNAP_SPECIES 8
typedef struct ipg_snap_params {
  int32_t twojmax;
  int32_t nspecies;
  double rcutfac;
  double rmin0;
  double rfac0;
  double radii[IPG_MAX_SNAP_SPECIES];
  double weight[IPG_MAX_SNAP_SPECIES];
  int32_t chem_flag;
  int32_t bzero_flag;
  int32_t bnorm_flag;
  int32_t switch_flag;
  int32_t wselfall_flag;
  int32_t literal_sqrt_radius; /* reproduce utl.jl:81's sqrt(cutmax) search radius */
  int32_t quadratic_flag;      /* quadratic SNAP                                       */
  int32_t literal_chem_z;      /* reproduce compute_z.jl:44-47's Z index with chem_flag */
} ipg_snap_params;

/* Builds the prebuilt tables of initialize_prebuilt_arrays (prebuilt_arrays.jl:48-247)
 * and uploads them.  The ctx must outlive the handle. */
IPG_API int ipg_snap_create(ipg_ctx* ctx, const ipg_snap_params* params, ipg_snap** out);
IPG_API int ipg_snap_destroy(ipg_snap* snap);
/* K = length(snap) = get_num_snap_coeffs (utl.jl:8-25). */
IPG_API int ipg_snap_ncoeff(const ipg_snap* snap, int32_t* K);

/* compute_local_descriptors / compute_force_descriptors / compute_all_descriptors
 * (src/BasisSystems/SNAP/snap.jl:103-124, 126-167, 226-285; the force descriptors follow
 * compute_all_descriptors' row indexing, snap.jl:261).
 *   B  [n][K]
 *   dB [n][K*nspecies][3]   (each atom's 3 x (K*nspecies) matrix, column-major)
 *   W  [K*nspecies][6]      (6 x (K*nspecies), column-major; absolute positions as in
 *                            snap.jl:267-281)                                          */
#define IPG_DESC_B 1u
#define IPG_DESC_DB 2u
#define IPG_DESC_W 4u
IPG_API int ipg_snap_descriptors(ipg_snap* snap, int64_t n, const double* pos, const int32_t* species, const double L[3],
                         double* B, double* dB, double* W, uint32_t what);

/* potential_energy / force / energy_and_force / virial_stress of LBasisPotential over
 * SNAP (src/BasisPotentials/basis_potentials.jl:14-57, linear_potential.jl:20-49):
 *   E = beta0 + sum_i beta[s_i] . B_i,  F_k = sum_blocks dB_k[:, block] . beta[block],
 *   W6 = W . beta.
 * beta is [nspecies][K] (one block per centre species; the reference's single K-vector
 * is every block equal).  mode IPG_SNAP_PLAIN materialises every per-neighbor dB/dr
 * and contracts it; IPG_SNAP_ADJOINT accumulates Y = d(beta.B)/dU per atom and
 * contracts dU/dr with Y per neighbor (design of compute_yi.jl / compute_dij.jl).     */
#define IPG_SNAP_PLAIN 0
#define IPG_SNAP_ADJOINT 1
IPG_API int ipg_snap_energy_forces(ipg_snap* snap, int64_t n, const double* pos, const int32_t* species, const double L[3],
                           const double* beta, double beta0, int32_t mode, double* E, double* F, double* W6);
IPG_API int ipg_snap_energy_forces_dev(ipg_snap* snap, int64_t n, const double* d_pos, const int32_t* d_species,
                               const double L[3], const double* beta, double beta0, int32_t mode, double* d_E,
                               double* d_F, double* d_W6);

/* Vector-Jacobian product of (E, F) with respect to beta (the pullback of the
 * ChainRulesCore.rrule for potential_energy / force):
 *   gbeta[s][k] = gE * sum_{i: s_i=s} B_i[k] + sum_atoms gF_atom . dB_atom[:, block s][k],
 *   gbeta0 = gE.  gF [3n] may be NULL (energy-only pullback).                          */
IPG_API int ipg_snap_vjp_beta(ipg_snap* snap, int64_t n, const double* pos, const int32_t* species, const double L[3],
                      double gE, const double* gF, double* gbeta, double* gbeta0);

/* Full pullback of (E, F) (the ChainRulesCore.rrule of energy_and_force / potential_energy
 * for LBasisPotential over SNAP): cotangents gE of E and gF [3n] of F (NULL = 0) give
 *   gbeta [nspecies][K] and gbeta0 as ipg_snap_vjp_beta, and
 *   gpos [3n] = d(gE E + gF . F)/dpos = -gE F - H gF    (H: Hessian of E).
 * Both terms are exact: F from one adjoint evaluation, H gF as the directional derivative of
 * the adjoint force computation along gF (the second-order extension of compute_dij.jl:5-74):
 * the tangent of Utot (the beta pullback's V kernel), the tangent of Y by polarization of the
 * quadratic form Y(Utot) (two Y evaluations at Utot +/- s Utot_dot, s a power of two; no
 * truncation term), and forward-mode tangents through the Wigner recursion and dE/dr per pair.
 * Environment IPG_GENERIC_HVP=1 at ipg_snap_create selects the per-atom kernel that carries
 * every phase in forward mode instead (same results to rounding).  Any of gbeta, gbeta0, gpos
 * may be NULL; beta [nspecies][K] is needed for gpos.  twojmax above 8 returns
 * IPG_ERR_UNSUPPORTED for gpos.  The reference
 * defines no rrule; this is the pullback that Zygote / ChainRules callers of
 * energy_and_force(s, lbp) need.                                                          */
IPG_API int ipg_snap_vjp(ipg_snap* snap, int64_t n, const double* pos, const int32_t* species, const double L[3],
                 const double* beta, double gE, const double* gF, double* gbeta, double* gbeta0, double* gpos);

/* Autotuner: times the adjoint evaluation of this configuration under each candidate kernel
 * configuration and keeps the fastest for the handle.  Coordinate descent over the Y kernel
 * (row-blocked or one Z entry at a time: the twojmax-dependent shared-memory layout), the
 * per-neighbor kernel (all chains of a pair per thread, or one chain per thread), the Utot
 * kernel (all chains in one launch, or one launch per chain with 1, 2 or 4 atoms per block)
 * and the atoms (warps) per block of the neighbor walk (1, 2, 4).  cache_path
 * (optional): a JSON-lines file keyed by device, twojmax, nspecies and the atom count
 * rounded up to a power of two; a hit applies the stored choice without timing, a miss
 * appends the result.  report (optional) receives the choice as one JSON object.        */
IPG_API int ipg_snap_autotune(ipg_snap* snap, int64_t n, const double* pos, const int32_t* species, const double L[3],
                      const double* beta, const char* cache_path, char* report, int32_t report_len);

/* Neighbor-list reuse across calls, for MD loops (the Verlet skin that nnlist.jl:1 leaves to
 * a future neighbor package): with skin > 0 the full SNAP list is built with every cutoff
 * enlarged by `skin` and kept in the handle; later calls with the same atom count,
 * configuration offsets and boxes take their pairs from it (re-measured at the current
 * positions with the same inclusion test as a fresh build) until some atom has moved more
 * than skin/2 since the build, a species id differs from the one at the build (the enlarged
 * cutoffs depend on the species pair) or a position is not finite; any of these rebuilds it,
 * so bad inputs are reported as by a fresh build.  Results equal those of a fresh build up
 * to the order of summation.  skin = 0 (the default) builds every call; graph replays and
 * the literal search radius always build.  ipg_snap_skin_stats counts builds and reuses.  */
IPG_API int ipg_snap_set_skin(ipg_snap* snap, double skin);
IPG_API int ipg_snap_skin_stats(const ipg_snap* snap, int64_t* builds, int64_t* reuses);

/* Fitting matrices of many configurations (the linear system A beta = b that
 * PotentialLearning solves; the row layout of get_snap, LAMMPS_SNAP/bispectrum.jl:279-387,
 * with one column per species block and component, col = s*K + k):
 *   Ae [nconfig][K*nspecies]     energy rows: sum of B_i over the atoms of species s
 *                                (E_c = Ae[c] . beta + beta0)
 *   Af [3 n_total][K*nspecies]   force rows: row 3a + x is dB_a[x][:] (F_a,x = Af[3a+x] . beta)
 *   Aw [nconfig][6][K*nspecies]  virial rows (W of compute_all_descriptors, snap.jl:267-281)
 * Atoms as in ipg_snap_batch_energy_forces; any of Ae, Af, Aw may be NULL.  The per-pair
 * dB/dr of the whole batch is materialised on the device (K*3 doubles per directed pair). */
IPG_API int ipg_snap_batch_descriptors(ipg_snap* snap, int32_t nconfig, const int64_t* atom_offsets,
                                       const double* pos, const int32_t* species, const double* L, double* Ae,
                                       double* Af, double* Aw);

/* ---- batched SNAP ------------------------------------------------------------------------
 * Many configurations at once: atoms of configuration c are atom_offsets[c] ..
 * atom_offsets[c+1]-1 of the flattened arrays; L is [nconfig][3].  Per-configuration
 * energies E [nconfig] (each with beta0) and virials W6 [nconfig][6]; forces [3 n_total].
 * _dev with graph != 0: the first call runs eagerly and then captures the evaluation
 * (neighbor build included) into a CUDA graph; later calls with the same atom_offsets,
 * boxes, mode and device buffers replay it with one graph launch (new positions, species
 * and beta are read from the buffers).  The captured pair buffers have 25% headroom over
 * the pair count seen at capture; a replay that needs more re-runs eagerly and
 * recaptures.  Configurations with an open axis (L = INFINITY) always run eagerly.      */
IPG_API int ipg_snap_batch_energy_forces(ipg_snap* snap, int32_t nconfig, const int64_t* atom_offsets, const double* pos,
                                 const int32_t* species, const double* L, const double* beta, double beta0,
                                 int32_t mode, double* E, double* F, double* W6);
IPG_API int ipg_snap_batch_energy_forces_dev(ipg_snap* snap, int32_t nconfig, const int64_t* atom_offsets,
                                     const double* d_pos, const int32_t* d_species, const double* L,
                                     const double* beta, double beta0, int32_t mode, int32_t graph, double* d_E,
                                     double* d_F, double* d_W6);
/* Force-matching loss over a batch, L = sum_atoms |F - F_ref|^2, with its gradient with
 * respect to beta [nspecies][K] (gradient of beta0 is 0).  F_ref [3 n_total].         */
IPG_API int ipg_snap_batch_loss_grad(ipg_snap* snap, int32_t nconfig, const int64_t* atom_offsets, const double* pos,
                             const int32_t* species, const double* L, const double* beta, double beta0,
                             const double* F_ref, double* loss, double* gbeta);
/* One training step of force matching on device buffers: E [nconfig], F [3 n_total] (required),
 * W6 [nconfig][6] (E and W6 may be NULL), the loss L = sum |F - F_ref|^2 [1] and dL/dbeta
 * [nspecies][K], from one adjoint evaluation whose pair list, Utot and Z the beta pullback
 * reuses.  The pullback of the force-matching loss through LBasisPotential's forces
 * (src/BasisPotentials/linear_potential.jl:37-49) over the fitting rows of
 * src/BasisSystems/LAMMPS_SNAP/bispectrum.jl:279-387; the reference evaluates it only by
 * assembling the dB matrix.  graph != 0: as ipg_snap_batch_energy_forces_dev, the whole step
 * (neighbor build, evaluation, loss, gradient) is captured on the first call and later calls
 * with the same offsets, boxes and buffers replay it with one graph launch.               */
IPG_API int ipg_snap_batch_loss_grad_dev(ipg_snap* snap, int32_t nconfig, const int64_t* atom_offsets,
                                         const double* d_pos, const int32_t* d_species, const double* L,
                                         const double* beta, double beta0, const double* d_F_ref, int32_t graph,
                                         double* d_E, double* d_F, double* d_W6, double* d_loss, double* d_gbeta);

#ifdef __cplusplus
}
#endif

#endif /* IPG_H */
