/*
 * qd_imsrg.h -- C ABI of the B200-native IM-SRG(2) commutator engine.
 *
 * Drop-in boundary for the commutator / BCH hot path of nparz/qd_IMSRG.
 * Each entry point below names the reference subroutine it replaces
 * (file:line inside the reference project).  The Fortran host keeps
 * Hartree-Fock, TBME generation and EOM; it hands the normal-ordered
 * Hamiltonian to this library in the reference's own flat "vectorize" order
 * (src/ME_general.f90:1871-1989) and calls the commutator / BCH / Magnus
 * routines on device-resident operators, through an iso_c_binding interface
 * module on the Fortran side.
 *
 * Conventions
 *   - Every function returns an int status: QD_OK (0) or a QD_ERR_* code;
 *     qd_last_error() gives a message for the calling thread.  (The
 *     reference has no error returns; it STOPs.)
 *   - Operators live in device memory owned by the library, one flat FP64
 *     array per operator in vectorize order: E0, fhh(n,n), fpp(m-n,m-n),
 *     fph(m-n,n), then per (M_L,M_S) block Vhhhh, Vpppp, Vpphh, Vphph,
 *     Vppph, Vphhh, each column-major.  herm (+1 Hermitian, -1
 *     anti-Hermitian) is a field of the operator, as full_ham%herm.
 *   - All work of one layout runs in order on that layout's CUDA stream.
 *     Calls on one layout are not reentrant.  Scalar results (energies,
 *     norms) synchronise the stream before returning.
 *   - Single-particle indices are in the reference's "states order"
 *     (arrange_states, src/ME_general.f90:688-716); holes must be states
 *     1..N (convertF, src/ME_general.f90:1517-1525).
 */
#ifndef QD_IMSRG_H
#define QD_IMSRG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QD_OK 0
#define QD_ERR_ARG 1        /* bad argument (null handle, size mismatch, ...) */
#define QD_ERR_LAYOUT 2     /* layout cannot be built (holes not states 1..N) */
#define QD_ERR_CUDA 3       /* a CUDA call failed                              */
#define QD_ERR_OOM 4        /* device allocation failed                        */
#define QD_ERR_NAN 5        /* non-finite value detected                       */
#define QD_ERR_NOCONV 6     /* flow did not converge within the step limit     */
#define QD_ERR_NODEVICE 7   /* no CUDA device / extension unusable             */
#define QD_ERR_STATE 8      /* call order violated (e.g. no cross-coupled data) */

typedef struct qd_layout qd_layout; /* basis + (M_L,M_S) block layout           */
typedef struct qd_op qd_op;         /* one operator: type(full_ham) on device    */
typedef struct qd_cc qd_cc;         /* one type(cc_mat): Pandya X(r,nb) matrices */

const char* qd_last_error(void);
const char* qd_version(void);

/* ---- layout: arrange_states + reindex + build_cross_coupled --------------
 * Replaces src/ME_general.f90:688-716 (arrange_states), :956-1116
 * (reindex), :363-448 (build_cross_coupled) and :1755-1778
 * (get_num_elements).  eig: m single-particle energies in states order
 * (m = emax*(emax+1)), or NULL for oscillator energies 2n+|ml|+1; pairs are
 * classed hole/particle by eig <= eF exactly as reindex does.
 * device >= 0 selects a CUDA device, -1 keeps the current device, and
 * QD_HOST_ONLY builds the host-side tables only (no CUDA calls; operators
 * cannot be created on such a layout, but qd_layout_* queries and
 * qd_random_operator work).  */
#define QD_HOST_ONLY (-2)
int qd_layout_create(int nbody, int emax, const double* eig, int device, qd_layout** out);
int qd_layout_destroy(qd_layout* L);
int qd_layout_info(const qd_layout* L, int* nbody, int* msp, int* nblock, int64_t* neq, int* ncc);
/* per block q (0-based): nhh, nph, npp, ML, MS  (5 ints per block)          */
int qd_layout_blocks(const qd_layout* L, int* dims5);
/* per block: vectorize offsets of Vhhhh,Vpppp,Vpphh,Vphph,Vppph,Vphhh      */
int qd_layout_offsets(const qd_layout* L, int64_t* off6);
/* pair list of block q (0-based), kind 0=hh 1=ph 2=pp; 1-based states,
 * (count x 2) row-major; returns the count in *count                        */
int qd_layout_pairs(const qd_layout* L, int q, int kind, int* out, int* count);
/* CUDA stream (cudaStream_t) used for this layout; NULL = library-owned    */
int qd_layout_set_stream(qd_layout* L, void* stream);
/* Precision of the block contractions (the dgemm calls of matrix_mult222,
 * construct_cc_ints, commutator_221 and commutator_111) on this layout:
 * slices = 0 plain FP64 (the reference's arithmetic), 1..8 the split form of
 * qd_gemm_split with that many BF16 slices per operand.  Everything else
 * (one-body, 122, 121, 221 traces, Pandya gathers, E0, norms, BCH sums, HF)
 * stays FP64.  No reference counterpart (the reference is FP64 only).       */
int qd_layout_set_split(qd_layout* L, int slices);
/* BCH terms (qd_bch_expand, and the flows built on it) as CUDA graphs: a
 * term seen before with the same buffers, zero-part masks, herm, flags and
 * coefficient is captured once and replayed with one launch (default on;
 * the stage profiler bypasses it).  Results are identical either way.
 * qd_layout_graph_stats: graphs captured and replays so far.               */
int qd_layout_set_graphs(qd_layout* L, int enable);
int qd_layout_graph_stats(const qd_layout* L, int64_t* captured, int64_t* replays);
int qd_layout_get_split(const qd_layout* L, int* slices);
int qd_layout_synchronize(qd_layout* L);
/* device bytes currently held by the layout's work arena                    */
int qd_layout_workspace_bytes(const qd_layout* L, int64_t* bytes);
/* Optional per-stage timing with CUDA events on the layout's stream (the
 * reference only has omp_get_wtime around whole runs, magnus_IMSRG.f90:30,159).
 * enable != 0 starts (and resets) it.  qd_layout_profile_read synchronises
 * and returns accumulated milliseconds and launch counts per stage:
 * 0 E0 (110+220), 1 commutator_111, 2 commutator_121, 3 commutator_221,
 * 4 commutator_122, 5 calc_cc, 6 ladder GEMMs (matrix_mult222),
 * 7 Pandya GEMMs (construct_cc_ints), 8 particle-hole gather, 9 BCH glue.  */
#define QD_NSTAGE 10
int qd_layout_profile(qd_layout* L, int enable);
int qd_layout_profile_read(qd_layout* L, double* ms, int64_t* counts, int nstage);
/* number of kernels this library has launched for the layout so far        */
int qd_layout_launches(const qd_layout* L, int64_t* n);
/* The autotuner's choices so far, as text: the first commutator_122 launch
 * for each pair of zero-part masks times every launch bucket with 128- and
 * 256-thread CTAs and keeps the faster (results do not depend on it).
 * Writes at most len bytes (NUL-terminated) into buf; *needed = full size.
 * No reference counterpart.                                                 */
int qd_layout_tuning(const qd_layout* L, char* buf, int64_t len, int64_t* needed);

/* ---- operators: allocate_everything / vectorize / repackage ---------------
 * Replaces src/IMSRG_tools.f90:465-537 (allocate_everything: zero-filled,
 * herm = herm), src/ME_general.f90:1871-1989 (vectorize) and :1992-2109
 * (repackage).                                                               */
int qd_op_create(qd_layout* L, int herm, qd_op** out);
int qd_op_destroy(qd_op* op);
int qd_op_upload(qd_op* op, const double* host_vec, int64_t neq);
int qd_op_download(const qd_op* op, double* host_vec, int64_t neq);
/* device <-> device in vectorize order (pointers into device memory)        */
int qd_op_upload_device(qd_op* op, const double* dev_vec, int64_t neq);
int qd_op_set_herm(qd_op* op, int herm);
int qd_op_get_herm(const qd_op* op, int* herm);
/* raw device pointer of the operator's array (for interop, e.g. torch)     */
int qd_op_device_ptr(qd_op* op, double** dptr);
/* Seeded random operator in vectorize order, written to a host buffer:
 * entries iid N(0, sigma^2) (Philox-4x32-10 counter RNG, Box-Muller),
 * diagonal-class blocks (fhh,fpp,Vhhhh,Vpppp,Vphph) made (X + herm X^T)/2,
 * E0 = 0; conserve != 0 zeroes one-body entries that change (ml,ms).
 * No counterpart in the reference (synthetic input generator).              */
int qd_random_operator(const qd_layout* L, int herm, uint64_t seed, double sigma, int conserve,
                       double* host_vec, int64_t neq);

/* ---- algebra (src/ME_general.f90:592-686, :2112-2138) ---------------------- */
int qd_add_arrays(const qd_op* r1, double s1, const qd_op* r2, double s2, qd_op* r3); /* r3=s1*r1+s2*r2 */
int qd_copy_arrays(const qd_op* r1, qd_op* r2);                                        /* r2 = r1      */
int qd_set_to_zero(qd_op* r1);
/* mat_2_norm (:2112-2138): sqrt of the sum of squares of every stored one-
 * and two-body entry, E0 excluded: fph, fpp, fhh and, per block, Vhhhh,
 * Vpppp, Vpphh, Vphph, Vphhh, Vppph.  Synchronous.                          */
int qd_mat_2_norm(const qd_op* r, double* out);

/* Allocation-free mat_2_norm, for callers that must not allocate device
 * memory while they run (a host that reserves its device-memory budget up
 * front and forbids allocation inside its flow loop, or one whose memory is
 * held by another allocator, where cudaMalloc may fail or synchronise the
 * device).  Same value as qd_mat_2_norm (every stored one- and two-body
 * entry); no counterpart in the reference.
 *   d_op   device array of one operator of layout L in vectorize order (e.g.
 *          from qd_op_device_ptr); d_norm: device double receiving the norm;
 *   stream cudaStream_t to run on.  NULL: the layout's own stream, so the
 *          call is ordered after every earlier call on the layout and before
 *          every later one.  A caller's stream must be ordered against the
 *          layout's stream by the caller (qd_layout_synchronize, or events).
 *          The call is asynchronous: d_norm holds the norm once the stream
 *          reaches it.
 * Nothing is allocated: the partial sums live in a static device array of
 * QD_NOALLOC_MAX_PARTIALS doubles (32 KiB, held by every GPU that loads the
 * library until exit).  Layouts with more than QD_NOALLOC_MAX_ENTRIES one-
 * and two-body entries (1 GiB per operator) are rejected with QD_ERR_ARG.
 * The kernels run on the layout's device; the calling thread's current
 * device is restored before returning.  The first call on a device looks up
 * the array's device address (cudaGetSymbolAddress); make that first call
 * before any stream capture.  All calls share the array, so calls that
 * overlap on the GPU race.                                                   */
#define QD_NOALLOC_MAX_PARTIALS 4096
#define QD_NOALLOC_MAX_ENTRIES (4096LL * 32768LL)
int qd_mat_2_norm_noalloc(const qd_layout* L, const double* d_op, double* d_norm, void* stream);

/* ---- commutators (src/commutators.f90) ------------------------------------- */
int qd_commutator_110(const qd_op* r1, const qd_op* r2, double* c);  /* :12-33   */
int qd_commutator_220(const qd_op* r1, const qd_op* r2, double* c);  /* :36-70   */
int qd_commutator_111(const qd_op* r1, const qd_op* r2, qd_op* r3);  /* :137-195, overwrites 1-body */
int qd_commutator_121(const qd_op* r1, const qd_op* r2, qd_op* r3);  /* :73-134, accumulates 1-body */
int qd_commutator_221(const qd_op* r1, const qd_op* r2, qd_op* r3, qd_op* w1, qd_op* w2); /* :198-352 */
int qd_commutator_122(const qd_op* r1, const qd_op* r2, qd_op* r3);  /* :355-676, overwrites 2-body */
/* :679-985 with matrix_mult222 :987-1132 and construct_cc_ints
 * (src/ME_general.f90:923-952); accumulates 2-body.  HCC belongs to r2,
 * ETACC to r1.  A qd_cc that calc_cc never filled holds X = 0, so its
 * particle-hole terms vanish (as in run_magnus).  w1 is accepted for
 * interface parity and is not used.                                          */
int qd_commutator_222(const qd_op* r1, const qd_op* r2, qd_op* r3, qd_op* w1, const qd_cc* HCC,
                      const qd_cc* ETACC);

/* Whole [A,B] -> C in the reference's order (E0 = 110+220; 111; 121; 221;
 * 122; 222).  flags: QD_PANDYA = fill both operators' cross-coupled
 * matrices first (as dGam, src/gs_IMSRG.f90:243-250); without it the
 * particle-hole channel is skipped (X = 0, as run_magnus).                  */
#define QD_PANDYA 1u
int qd_commutator(const qd_op* A, const qd_op* B, qd_op* C, unsigned flags);
/* dGam, src/gs_IMSRG.f90:223-273: the derivative of the ODE form of the flow,
 * the right-hand side the host's Adams integrator (adams_ode) evaluates.
 * ETA = build_white(H) on a zeroed generator (herm -1), HCC = calc_cc(H),
 * ETACC = calc_cc(ETA), DER = [ETA, H] with all terms including the
 * particle-hole channel.  HCC / ETACC are filled as in the reference (NULL:
 * library workspaces).  The reference's vectorize(DER, yp) is
 * qd_op_download(DER, yp, neq); its repackage(H, y) is qd_op_upload.        */
int qd_dgam(const qd_op* H, qd_op* DER, qd_cc* HCC, qd_cc* ETACC);
/* EOM matrix-vector product for the scalar target (M_L, M_S) = (0, 0):
 * matvec_prod (src/EOM_IMSRG.f90:551-649) with HQ_comm_1b / HQ_comm_2b
 * (src/commutators.f90:1162-1272).  Q's fph and Vpphh hold the 1p1h and 2p2h
 * amplitudes (its other parts are ignored); HQ receives fph = HQ_comm_1b and
 * Vpphh = HQ_comm_2b, every other part zero.  Computed as the particle-hole
 * and pphh parts of ([H, Q+] + [H, Q-]) / 2 with Q+- the amplitudes as
 * herm +-1 operators (particle-hole channel on).  The Lanczos driver
 * (ARPACK dsaupd) stays on the host, as in the reference; its vector maps to
 * Q through the host's unwrap/rewrap.  Any target, non-scalar ones included:
 * qd_eom_matvec_target.                                                     */
int qd_eom_matvec(const qd_op* H, const qd_op* Q, qd_op* HQ);
/* EOM vector dimension for the target (ml, ms) (Mltarg, Mstarg of the
 * reference, src/EOM_IMSRG.f90:21-22: Ml = m_l(a) - m_l(i), Ms = s(a) - s(i)
 * with s = +-1): *n1 1p1h and *n2 2p2h entries, counted as unwrap
 * (src/EOM_IMSRG.f90:815-884) counts them.  Host only; works on QD_HOST_ONLY
 * layouts.                                                                  */
int qd_eom_dim(const qd_layout* L, int ml, int ms, int64_t* n1, int64_t* n2);
/* matvec_prod (src/EOM_IMSRG.f90:551-649) for any target (ml, ms): d_w = the
 * rewrap of HQ_comm_1b / HQ_comm_2b (src/commutators.f90:1162-1272) of H and
 * the excitation operator unwrapped from d_v.  d_v and d_w are device arrays
 * of n = n1 + n2 doubles in the reference's unwrap order (1p1h entries,
 * particle outer and hole inner, then 2p2h entries, a < b outer and i < j
 * inner); the ARPACK loop (dsaupd reverse communication,
 * src/EOM_IMSRG.f90:243-255) stays on the host and copies its work vectors
 * to and from them.  Asynchronous on the layout's stream.  The first call
 * for a target builds its tables (and synchronises); they are kept until
 * the layout is destroyed.  Returns QD_ERR_ARG when n does not match the
 * target's dimension.                                                       */
int qd_eom_matvec_target(const qd_op* H, int ml, int ms, const double* d_v, double* d_w, int64_t n);

/* ---- cross-coupled (Pandya) matrices ----------------------------------------
 * calc_cc src/commutators.f90:1135-1159, copy_cc src/IMSRG_tools.f90:437-461 */
int qd_cc_create(qd_layout* L, double herm, qd_cc** out);  /* X = 0 */
int qd_cc_destroy(qd_cc* cc);
int qd_cc_set_herm(qd_cc* cc, double herm);
int qd_calc_cc(const qd_op* H, qd_cc* HCC);
int qd_cc_download(const qd_cc* cc, double* host, int64_t n, int64_t* needed);

/* ---- generator, energies ---------------------------------------------------- */
int qd_build_white(qd_op* gen, const qd_op* H);  /* src/IMSRG_tools.f90:377-434 */
int qd_mbpt2(const qd_op* H, double* out);        /* src/HFQDmod.f90:325-362   */
/* HF_E2, src/HFQDmod.f90:292-323: E0 = sum_{i<=N} eig(i) - sum Vhhhh(j,j);
 * sets H's E0 as the reference does (eig as given to qd_layout_create)       */
int qd_hf_e2(qd_op* H, double* out);

/* ---- host-side inputs: Coulomb TBMEs and Hartree-Fock -----------------------
 * The reference computes these on the host (generate_ME.f90, get_TBME.f90,
 * src/HFQDmod.f90:9-254); they are the flow's input, not its hot path.       */
/* TBME options.  QD_TBME_QUAD: evaluate v_int with every sum and factor in
 * __float128.  The reference's arithmetic sums terms of up to ~1e21 in
 * real(8) and loses every digit from radial quantum number n ~ 7 on
 * (emax >= 15), so emax = 20 inputs need this option; without it v_int is
 * the reference's, rounding included.                                       */
#define QD_TBME_QUAD 1u
/* Write ME.bin (records int32 n1,m1,n2,m2,n3,m3,n4,m4 + float64 Vdir at
 * hbar-omega = 1, the stream read at src/HFQDmod.f90:97-127) for every
 * m-conserving quadruple of spatial orbitals below emax shells, from v_int
 * (src/ME_general.f90:2205-2276).  nthreads <= 0: 1.  options: QD_TBME_QUAD. */
int qd_tbme_write(int emax, const char* path, int nthreads, unsigned options);
/* construct_two_particle_HF_BASIS + HF_E2: HF single-particle energies (eig,
 * m = emax*(emax+1), states order) and the normal-ordered HF Hamiltonian in
 * vectorize order (vec, neq entries; E0 = E_HF).  mebin: ME.bin path, or NULL
 * to compute the TBMEs in memory (options: QD_TBME_QUAD).  mix: fraction of
 * the new density per iteration (1 = the reference's plain iteration, which
 * oscillates for e.g. N=20 at hbar-omega=0.5; 0.5 damps it).
 * *iterations: HF iterations.                                               */
int qd_hf_hamiltonian(int nbody, int emax, double hw, const char* mebin, int nthreads, double mix,
                      unsigned options, double* eig, double* vec, int64_t neq, int* iterations);
/* v_int(qi,qj,qk,ql,hw) with q = (n, ml, ms) (src/ME_general.f90:2205), in
 * the reference's arithmetic; qd_v_int_quad in __float128 throughout.       */
double qd_v_int(const int* qi, const int* qj, const int* qk, const int* ql, double hw);
double qd_v_int_quad(const int* qi, const int* qj, const int* qk, const int* ql, double hw);

/* ---- BCH / Magnus (src/magnus_IMSRG.f90) ----------------------------------- */
/* BCH_EXPAND :253-318: HS = sum_k ad_G^k(H) cof(k) with the reference's
 * truncated cof table and exit test mat_2_norm(INT2)*cof/mat_2_norm(INT1)
 * < 1e-5.  INT2, AD, w1, w2 are caller workspaces (contents unspecified on
 * return).  INT1 is not written: the reference copies HS into it before
 * every term (:290) only to take its norm, which is taken here from HS in
 * the same pass as the update; a caller that reads INT1 afterwards must copy
 * HS itself.  HCC/OCC as in the reference (never filled -> no ph channel)
 * unless flags has QD_PANDYA, which refills them from AD and G before each
 * 222.  *nterms receives the number of commutators evaluated.               */
int qd_bch_expand(qd_op* HS, const qd_op* G, const qd_op* H, qd_op* INT1, qd_op* INT2, qd_op* AD,
                  qd_op* w1, qd_op* w2, qd_cc* HCC, qd_cc* OCC, unsigned flags, int* nterms);
/* MAGNUS_EXPAND :321-369: the reference returns after DG = ETA.              */
int qd_magnus_expand(qd_op* DG, const qd_op* G, const qd_op* ETA);
/* euler_step :372-384: G = G + stp*DG; s = s + stp                          */
int qd_euler_step(qd_op* G, const qd_op* DG, double* s, double stp);

/* s_evolve with build_white, :194-248 (TDA diagnostics omitted).  HAM is the
 * normal-ordered HF Hamiltonian, HS receives the evolved Hamiltonian.
 * trace (may be NULL): up to max_iter rows of 7 doubles per flow iteration:
 * iteration, s, E0, nrm1, nrm2, crit, BCH terms (negated for a rejected
 * step).  *rows = rows written.  Returns QD_ERR_NOCONV past max_iter.      */
typedef struct qd_flow_result {
  double E0;        /* HS%E0 at convergence                  */
  double s;         /* final flow parameter                  */
  int iterations;   /* accepted steps                        */
  int rejected;     /* rejected steps                        */
  int commutators;  /* total BCH commutators evaluated       */
  int rows;         /* trace rows written                    */
} qd_flow_result;
int qd_magnus_flow(const qd_op* HAM, qd_op* HS, unsigned flags, int max_iter, double* trace,
                   qd_flow_result* result);
/* The same flow as a stepping object, for callers that inspect or seed
 * Omega (no reference counterpart: run_magnus owns its loop).  One flow per
 * layout at a time (its workspaces are the layout's).
 *   qd_flow_create      s = 0: HS = HAM, ETA = build_white(HS), nrm1 = |ETA|
 *   qd_flow_warm_start  Omega = G at flow parameter s: HS = BCH(G, HAM),
 *                       ETA = build_white(HS); nrm1 keeps its s = 0 value
 *   qd_flow_step        one pass of s_evolve's loop (accepted or rejected)
 *   qd_flow_omega       the flow's current Omega (owned by the flow)       */
typedef struct qd_flow qd_flow;
typedef struct qd_flow_step_info {
  double s, E0, nrm1, nrm2, crit;  /* crit: |MBPT2| before the step        */
  int terms;                       /* BCH commutators of the step           */
  int accepted;                    /* 0: rejected on eta-norm growth        */
  int converged;                   /* |MBPT2(HS)| <= 1e-9 after the step    */
} qd_flow_step_info;
int qd_flow_create(const qd_op* HAM, qd_op* HS, unsigned flags, qd_flow** flow);
int qd_flow_warm_start(qd_flow* flow, const qd_op* G, double s);
int qd_flow_step(qd_flow* flow, qd_flow_step_info* info);
int qd_flow_omega(const qd_flow* flow, qd_op** G);
int qd_flow_state(const qd_flow* flow, qd_flow_result* result);
int qd_flow_destroy(qd_flow* flow);
/* Several independent flows (e.g. a grid of (N, hbar-omega, emax)), one per
 * layout.  Default: the instances advance in lockstep on one stream, and each
 * BCH term's commutator_122 tiles and ladder GEMM tasks of every instance
 * whose series is still running go into one launch per kernel (uneven blocks
 * of all instances in one task list, longest first); the small stages run
 * per instance.  flags | QD_BATCH_STREAMS instead runs one host thread per
 * instance on its own layout's stream (each flow as qd_magnus_flow, BCH steps
 * as graphs).  Results equal the separate flows'.  No reference counterpart
 * (the reference runs one flow per process).  status[i] is instance i's
 * code; the call returns the first failing one (and names the instance in
 * qd_last_error).                                                           */
#define QD_BATCH_STREAMS 4u
int qd_magnus_flow_batch(int count, const qd_op* const* HAM, qd_op* const* HS, unsigned flags, int max_iter,
                         qd_flow_result* results, int* status);

/* ---- learned warm start (no reference counterpart) -------------------------
 * Omega of the White-generator flow is non-zero only in fph and Vpphh; its
 * "entries" are fph ((m-n) x n) followed by every block's Vpphh, in vectorize
 * order.  Device pointers (d_*) are the caller's.                           */
int qd_omega_count(const qd_layout* L, int64_t* n);
int qd_omega_gather(const qd_op* G, double* d_out, int64_t n);              /* d_out[e] = entry e of G */
/* G = 0 except entries e = scale * d_in[e] * (d_escale ? d_escale[e] : 1)    */
int qd_omega_scatter(qd_op* G, const float* d_in, float scale, const double* d_escale, int64_t n);
/* 16 float features per entry (16-byte aligned rows): energies of the four
 * legs and their occupations, the H element, hbar-omega, N, the channel
 * (M_L, M_S), the target flow parameter s, the shells and the entry kind.    */
int qd_omega_features(const qd_op* H, double hw, double s, float* d_X, int64_t n);

/* The per-entry network 16 -> 256 -> 256 -> 1 (GELU), FP32 master weights,
 * BF16 operands of the 256-wide layer on the tensor cores, FP32 accumulation.
 * Parameters: W1[256][16], b1[256], W2[256][256], b2[256], w3[256], b3.
 * qd_mlp_grad / qd_mlp_train_step: mean squared error over a batch whose size
 * is a multiple of 32; train_step = grad + one Adam step (lr).              */
#define QD_MLP_NPARAM 70401
typedef struct qd_mlp qd_mlp;
int qd_mlp_create(int device, uint64_t seed, qd_mlp** mlp);
int qd_mlp_destroy(qd_mlp* mlp);
int qd_mlp_get_params(const qd_mlp* mlp, float* host, int64_t n);
int qd_mlp_set_params(qd_mlp* mlp, const float* host, int64_t n);
int qd_mlp_forward(qd_mlp* mlp, const float* d_X, float* d_y, int64_t n, void* stream);
int qd_mlp_grad(qd_mlp* mlp, const float* d_X, const float* d_T, int64_t n, float* d_grad, float* loss, void* stream);
int qd_mlp_train_step(qd_mlp* mlp, const float* d_X, const float* d_T, int64_t n, float lr, float* loss,
                      void* stream);

/* ---- on-disk Hamiltonian: export_hamiltonian / import_hamiltonian --------
 * Replaces src/ME_general.f90:207-361.  The reference's Fortran unformatted
 * sequential file: one record per FP64 entry framed by 4-byte markers (8),
 * in its loop order (E0, fhh, fph, fpp row by row, then per block Vhhhh,
 * Vpppp, Vpphh, Vphph, Vphhh, Vppph row by row); no header.  The reference
 * prefixes '../hamiltonians/' to the name; `path` here is the full path.
 * qd_hamiltonian_write/read convert a host array in vectorize order (they
 * work on QD_HOST_ONLY layouts); qd_export/import_hamiltonian move a device
 * operator (download + write, read + upload).  A file whose size or record
 * markers do not match the layout is rejected with QD_ERR_ARG.             */
int qd_hamiltonian_write(const qd_layout* L, const double* vec, const char* path);
int qd_hamiltonian_read(const qd_layout* L, double* vec, const char* path);
int qd_export_hamiltonian(const qd_op* H, const char* path);
int qd_import_hamiltonian(qd_op* H, const char* path);

/* Split-precision FP64 product with dgemm's argument meaning (column-major;
 * transa/transb 'N' or 'T'): C = alpha op(A) op(B) + beta C on device arrays,
 * on the tcgen05 tensor cores.  Replaces the dgemm calls of matrix_mult222
 * (src/commutators.f90:987-1132) and construct_cc_ints
 * (src/ME_general.f90:923-952) in the split form.  Each row of op(A) and
 * column of op(B) is scaled by a power of two and cut into `slices` (1..8)
 * 7-bit integer BF16 slices; the slice products with s + t <= slices + 1 are
 * accumulated exactly in FP32 (TMEM) over K chunks and summed in FP64.  The
 * truncation error is about 2^(-7 slices) of max|row| max|column| K per
 * entry; slices = 8 reaches FP64 accuracy.  Synchronous on `stream`.       */
int qd_gemm_split(int device, void* stream, char transa, char transb, int M, int N, int K, double alpha,
                  const double* A, int lda, const double* B, int ldb, double beta, double* C, int ldc, int slices);

#ifdef __cplusplus
}
#endif
#endif /* QD_IMSRG_H */
