/*
 * mbforce.h -- C ABI of the B200 many-body force path (libmbforce.so).
 *
 * Plain pointers and sizes only.  Every array argument is DEVICE memory unless
 * its comment says "host"; `stream` is a cudaStream_t passed as void*.  The
 * library allocates nothing: callers pass workspaces sized by the *_bytes
 * queries.  Every function returns MBF_OK (0) or a negative MBF_ERR_* code;
 * mbf_error_string() names it.
 *
 * Each entry point replaces one interface of the reference (akitsushima
 * 0.4.0a4, Python + numba); the citation is given beside it.  The reference
 * has no native ABI of its own, so these functions are what a ctypes / cffi
 * binding from its Python layer would call.
 *
 * Units: A, eV, eV/A; the virial returned is sum over pairs of -f (x) r
 * (eV), NOT divided by the volume -- the caller divides, as the reference does
 * (engine/tersoff.py:1512, engine/eam.py:253).
 *
 * Layouts:
 *   positions  (n_atoms, 3) float64 row-major, Cartesian
 *   types      (n_atoms,)   int32 species index
 *   cells      (n_struct, 18) float64: lattice rows a0 a1 a2 (9), then the
 *              inverse lattice (9); cart = frac @ lattice
 *   struct_off (n_struct + 1) int32 atom offsets (atoms of structure s are
 *              struct_off[s] .. struct_off[s+1]-1); atom_struct (n_atoms,)
 *              int32 structure id of each atom
 *   grids      (n_struct, 8) int32: nc0 nc1 nc2, first global cell, and the
 *              per-axis stencil widths (1 if nc == 1, 2 if nc == 2, else 3)
 *   neighbour list: two-way CSR, row_off (n_atoms + 1) int32, nbr (n_slots)
 *              int32 with every row sorted ascending, rev (n_slots) int32 the
 *              slot of the reverse direction (rev[slot(a->b)] = slot(b->a)).
 */
#ifndef MBFORCE_H
#define MBFORCE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MBF_OK 0
#define MBF_ERR_ARGUMENT -1     /* bad size, null pointer or bad precision */
#define MBF_ERR_CUDA -2         /* a CUDA runtime call failed */
#define MBF_ERR_CAPACITY -3     /* nbr capacity too small; *n_slots holds the need */
#define MBF_ERR_ROW_TOO_LONG -4 /* a neighbour row exceeds the kernel's staging */
#define MBF_ERR_WORKSPACE -5    /* workspace too small */
#define MBF_ERR_SCRATCH_LIMIT -6 /* size beyond the no-allocation entry's limit */

#define MBF_FP64 0   /* all arithmetic in float64 */
#define MBF_MIXED 1  /* bond terms in float32; wrap, accumulation, EAM rho-bar in float64 */

typedef struct mbf_system {
    int n_atoms;
    int n_struct;
    const double *positions;   /* (n_atoms, 3) */
    const int *types;          /* (n_atoms,) */
    const int *atom_struct;    /* (n_atoms,) */
    const int *struct_off;     /* (n_struct + 1) */
    const double *cells;       /* (n_struct, 18) */
    int orthorhombic;          /* 1 if every lattice is diagonal (off-diagonal
                                  entries exactly 0): kernels use a 3-axis
                                  minimum image; 0 for general cells */
    const double *cells_host;  /* optional HOST copy of `cells` (n_struct, 18),
                                  equal to it, or NULL.  For one orthorhombic
                                  structure the mixed Zhou EAM evaluation then
                                  takes the cell as a launch argument (fewer
                                  registers, more resident warps) when the
                                  stream is not capturing; captured launches
                                  read `cells` at each replay. */
} mbf_system;

typedef struct mbf_nlist {
    int n_atoms;
    long long n_slots;
    int max_row;               /* host copy of the longest row */
    const int *row_off;        /* (n_atoms + 1) */
    const int *nbr;            /* (n_slots,) */
    const int *rev;            /* (n_slots,) */
    const int *upper;          /* (n_atoms,) first slot of row a whose neighbour is > a */
} mbf_nlist;

/* Per-structure reduction table: chunks of atoms that lie in one structure.
 * chunk (n_chunks, 3) int32 rows (struct id, first atom, end atom);
 * chunk_first (n_struct + 1) int32: chunks of structure s are
 * chunk_first[s] .. chunk_first[s+1]-1; a structure without atoms has one
 * empty chunk.  Any chunk length works; the last kernel of an evaluation runs
 * one block per chunk (8 threads per atom of the mean chunk, 128 to 512),
 * so chunks of 32-512 atoms, about two per SM, keep it busy. */
typedef struct mbf_reduce_plan {
    int n_chunks;
    const int *chunk;
    const int *chunk_first;
} mbf_reduce_plan;

const char *mbf_error_string(int code);
int mbf_version(void);

/* ---- neighbour list ---------------------------------------------------
 * Replaces NeighbourList.build / _build_cell_linked / _canonical_pair_order
 * (engine/neighborlist.py:574-585, :935-1024, :1166-1181) and the two-way CSR
 * every potential derives from it (engine/tersoff.py:1297-1307).  A pair
 * (a, b) is listed iff it lies in the cell stencil and r2 < r_list^2,
 * r2 > 1e-20, with r2 from the minimum-image displacement evaluated in the
 * reference's operation order without fused multiply-add
 * (engine/neighborlist.py:350-363), so the pair set equals the reference's
 * bit for bit.  n_cells_total = sum over structures of nc0*nc1*nc2.      */
size_t mbf_nl_workspace_bytes(int n_atoms, int n_cells_total);
/* The workspace with which mbf_nl_rebuild_async searches once instead of
 * twice: mbf_nl_workspace_bytes plus n_atoms x max_row_limit staging ints
 * (each row kept at a fixed stride during the count, then sorted into
 * the CSR).  A smaller workspace, of at least mbf_nl_workspace_bytes, runs
 * the count-then-fill search.                                            */
size_t mbf_nl_rebuild_workspace_bytes(int n_atoms, int n_cells_total, int max_row_limit);

/* Counts, scans and fills.  If nbr_capacity < the number of slots it stops
 * after the count, stores the need in *n_slots (host) and returns
 * MBF_ERR_CAPACITY; call again with a larger nbr/rev.  *n_slots and
 * *max_row are host outputs.  Synchronises `stream` once (to read the
 * count).  Workspace beyond mbf_nl_workspace_bytes serves as staging rows
 * (stride = the extra bytes / (4 n_atoms), at most 1024): when no row is
 * longer than that stride the search runs once, as in
 * mbf_nl_rebuild_async; size it with mbf_nl_rebuild_workspace_bytes and
 * a row bound estimate.  The list is the same either way. */
int mbf_nl_build(const mbf_system *sys, const int *grids, int n_cells_total,
                 double r_list, void *workspace, size_t workspace_bytes,
                 int *row_off, int *nbr, int *rev, int *upper, long long nbr_capacity,
                 long long *n_slots, int *max_row, void *stream);

/* Device status bits written by the graph-capturable entries below (OR-ed
 * into a caller-owned device int that the caller clears and reads). */
#define MBF_STATUS_ROW_TOO_LONG 1  /* a row beyond max_row_limit / staging */
#define MBF_STATUS_BAD_INDEX 2     /* an index check failed */
#define MBF_STATUS_CAPACITY 4      /* the list did not fit nbr_capacity */
#define MBF_STATUS_SKIN 8          /* a rebuild found the skin criterion broken */

/* The same list as mbf_nl_build rebuilt in place with no host
 * synchronisation, so it can be captured in a CUDA graph (the neighbour
 * list of a device MD loop, rebuilt at a fixed step interval).  The buffers
 * keep their addresses; the slot count stays on the device (row_off[n]).
 * A list that would need more than nbr_capacity slots, or a row longer than
 * max_row_limit (<= 1024), sets MBF_STATUS_CAPACITY / MBF_STATUS_ROW_TOO_LONG
 * in *status and leaves every row empty, so nothing is written out of
 * bounds.  No counterpart in the reference, whose lists are host arrays. */
int mbf_nl_rebuild_async(const mbf_system *sys, const int *grids, int n_cells_total,
                         double r_list, void *workspace, size_t workspace_bytes,
                         int *row_off, int *nbr, int *rev, int *upper,
                         long long nbr_capacity, int max_row_limit, int *status,
                         void *stream);

/* Largest minimum-image displacement of any atom from its reference
 * position mapped by the lattice change (engine/neighborlist.py:653-668):
 * writes max_i |MIC(r_i - r_ref_i @ M_s)| per structure to d_max (n_struct),
 * M_s = inv(lattice_build_s) @ lattice_now_s given per structure as
 * maps (n_struct, 9). */
int mbf_nl_max_displacement(const mbf_system *sys, const double *ref_positions,
                            const double *maps, double *d_max, void *stream);

/* Canonical half list (i < j sorted by (i, j), the reference's
 * get_candidate_pairs(), engine/neighborlist.py:679-714) extracted from the
 * two-way CSR: pair_i/pair_j sized n_slots / 2; the workspace needs
 * mbf_nl_half_workspace_bytes(n_atoms). */
size_t mbf_nl_half_workspace_bytes(int n_atoms);
int mbf_nl_half_pairs(const mbf_nlist *nl, int *pair_i, int *pair_j, void *workspace,
                      size_t workspace_bytes, void *stream);

/* ---- per-structure reduction workspace --------------------------------- */
/* Bytes of the workspace every *_eval below needs (per-atom accumulators,
 * per-slot three-body forces and bond orders, reduction partials). */
size_t mbf_eval_workspace_bytes(int n_atoms, long long n_slots, int n_chunks);

/* Status words of the last evaluation that used `workspace` (host_words[4],
 * synchronises `stream`): word 0 device error bits, word 1 the site of the
 * first failed index check (0 = none), word 2 the index that failed or the
 * atom whose row held it. */
int mbf_eval_status(const void *workspace, int *host_words, void *stream);

/* ---- EAM --------------------------------------------------------------
 * Replaces EAMPotential.compute's numba branch (engine/eam.py:174-256) and
 * _eam_kernel (engine/_eam_kernels.py:231-307): alloy EAM, rho-bar at an
 * atom from its neighbours' species densities, clamped at 0.
 * Function tables (device) as engine/_eam_kernels.py:77-121 lays them out:
 *   codes (nf,) int32: 1 spline, 2 spline/r, 3 Zhou density, 4 Zhou pair,
 *         5 Zhou cross pair, 6 Zhou embedding
 *   P     (nf, 43) float64 parameter rows; spline xo/nx (nf,) int32,
 *         X (nX,), C (4, nX).  A spline's P row may declare its knots
 *         uniform: P[0] = 1, P[1] = the first knot, P[2] = 1 / spacing
 *         (setfl tables are); its interval is then computed, not searched
 *         -- the same interval as searchsorted(side='right').  P row 0
 *         otherwise (binary search).
 *   rho_f, F_f (ns,) int32 and phi_f (ns, ns) int32 function ids.        */
typedef struct mbf_eam_tables {
    int ns;
    int nf;
    int nX;
    const int *codes;
    const double *P;
    const int *xo;
    const int *nx;
    const double *X;
    const double *C;
    const int *rho_f;
    const int *F_f;
    const int *phi_f;
    double r_cut;
    /* 1 when every function is a Zhou form (codes 3..6) sharing one switch
     * (r_c, width), each pair row holds its elements' density-row
     * parameters, and ns <= 8: the kernels then evaluate an element's
     * density and pair function from shared exponentials.  0: generic. */
    int zhou_fused;
    /* Optional HOST copies of P, rho_f and phi_f (all three, or NULL).  With
     * them a fused Zhou table of one or two elements runs its fastest path:
     * the element constants are passed as kernel arguments and both
     * elements are evaluated for every pair without a branch.  The copies
     * are read during the call only. */
    const double *P_host;
    const int *rho_f_host;
    const int *phi_f_host;
} mbf_eam_tables;

/* lanes_per_atom: lanes of one atom's group in the density and force
 * passes, 1, 2, 4 or 8 (0 = 8; other values: MBF_ERR_ARGUMENT). */
int mbf_eam_eval(const mbf_system *sys, const mbf_nlist *nl, const mbf_eam_tables *tab,
                 const mbf_reduce_plan *plan, int precision, int lanes_per_atom,
                 void *workspace, size_t workspace_bytes,
                 double *forces, double *energy, double *virial, void *stream);

/* The same evaluation in its two halves, for a structure split over ranks
 * (a slab per GPU with a halo of one list radius): the reference's phases 1-2
 * and 3-4 (engine/_eam_kernels.py:241-274 and :276-307).
 * mbf_eam_embedding runs the density and embedding passes and writes
 * F'(rho-bar) of every atom to fprime (n_atoms doubles, device).  The
 * owned atoms' values are exact; a halo atom's neighbourhood is cut, so
 * the caller replaces its F' by the value its owner computed.
 * mbf_eam_forces then takes that array, runs the force pass and the
 * gather, and writes forces, energy and virial as mbf_eam_eval does (the
 * reduction plan chooses whose records are summed).  Both calls use the
 * same workspace, list and tables; the workspace keeps rho-bar, F and the
 * positions between them.                                                 */
int mbf_eam_embedding(const mbf_system *sys, const mbf_nlist *nl, const mbf_eam_tables *tab,
                      const mbf_reduce_plan *plan, int precision, int lanes_per_atom,
                      void *workspace, size_t workspace_bytes, double *fprime, void *stream);
int mbf_eam_forces(const mbf_system *sys, const mbf_nlist *nl, const mbf_eam_tables *tab,
                   const mbf_reduce_plan *plan, int precision, int lanes_per_atom,
                   void *workspace, size_t workspace_bytes, const double *fprime,
                   double *forces, double *energy, double *virial, void *stream);

/* mbf_eam_eval without a workspace argument: no counterpart in the reference.
 * For callers that cannot allocate device memory -- a host program that
 * owns the whole device memory budget and gives its plug-ins only their
 * input and output buffers, or a time-step loop that must not pay the device
 * synchronisation cudaMalloc / cudaFree can cause.  The call allocates
 * nothing: its scratch is a fixed device array of
 * MBF_EAM_STATIC_SCRATCH_BYTES that the library reserves on every GPU that
 * loads it, until the process exits.  Inputs and outputs are as for
 * mbf_eam_eval.
 *   - Returns MBF_ERR_SCRATCH_LIMIT, doing nothing, when the structure needs
 *     more scratch than that (mbf_eval_workspace_bytes(n_atoms, n_slots,
 *     n_chunks) > MBF_EAM_STATIC_SCRATCH_BYTES, e.g. beyond about 8000 atoms
 *     of an fcc alloy with an 80-neighbour list).
 *   - The first call on a device looks the array's device address up (once
 *     per device); make that first call before any stream capture.
 *   - Every call on a device uses the same array and it keeps the previous
 *     call's contents (the call clears what must start at zero).  Calls whose
 *     work overlaps on the GPU -- two streams, or two host threads -- race
 *     on it: serialise them.                                              */
#define MBF_EAM_STATIC_SCRATCH_BYTES (32u << 20)
int mbf_eam_eval_static(const mbf_system *sys, const mbf_nlist *nl, const mbf_eam_tables *tab,
                        const mbf_reduce_plan *plan, int precision, int lanes_per_atom,
                        double *forces, double *energy, double *virial, void *stream);

/* The status words of the last mbf_eam_eval_static on the current device,
 * as mbf_eval_status gives them for a workspace (host_words[4]; synchronises
 * `stream`): the no-allocation entry's callers hold no workspace pointer,
 * so this is how they learn of a failed index check.  No counterpart in the
 * reference.                                                              */
int mbf_eam_eval_static_status(int *host_words, void *stream);

/* Zhou EAM adjoint for fitting: the vector-Jacobian product of (energy,
 * forces, virial) with respect to the function rows P (nf, 43) of an
 * analytic Zhou table (density rows code 3, embedding rows code 6, pair
 * rows code 4 / 5, as the table layout above), in float64.  Given upstream
 * gradients g_energy (n_struct), g_forces (n_atoms, 3) and g_virial
 * (n_struct, 9) -- any may be NULL for zero -- writes
 *   d_P[f, c] = sum_s gE_s dE_s/dP[f, c] + sum_a gF_a . dF_a/dP[f, c]
 *               + sum_s gW_s : dW_s/dP[f, c]
 * for the columns each row's function reads: density r_e, f_e, beta,
 * lambda; embedding rho_e, rho_s, Fn0..3, F0..3, eta, F_e; pair the element
 * columns of one (like) or both (cross) species and the cross factor
 * (column 42).  The switch columns 40, 41 and unread columns get 0.  The
 * derivative is of the float64 evaluation, with respect to the rows the
 * generic evaluation reads (rho_f, F_f, phi_f).  Replaces the
 * forward-difference Jacobian of the reference's fit over
 * ZhouEAMParameterSet (fitting/driver.py:802-816,
 * fitting/parameter_sets.py:1306-1400).  Each unordered pair is visited
 * once; deterministic.  ns <= 8; the workspace needs
 * mbf_eam_adjoint_workspace_bytes(n_atoms, n_slots, ns).                 */
size_t mbf_eam_adjoint_workspace_bytes(int n_atoms, long long n_slots, int ns);
int mbf_eam_adjoint(const mbf_system *sys, const mbf_nlist *nl, const mbf_eam_tables *tab,
                    const double *g_energy, const double *g_forces, const double *g_virial,
                    void *workspace, size_t workspace_bytes, double *d_P, void *stream);

/* ---- Tersoff ----------------------------------------------------------
 * Replaces TersoffPotential.compute (engine/tersoff.py:1208-1711): both the
 * single-species flat form (m = 3, gamma = 1; :1233-1513) and the
 * multi-species record form (:1518-1711), given as dense species tables
 * (:1606-1653).  tb (ns*ns, 10) float64 rows [valid, A, B, lambda1, lambda2,
 * R, D, beta, n, unused]; tri (ns*ns*ns, 8) rows [valid, c, d, h, lambda3,
 * m, gamma, unused]. r_cut = the largest R + D.                           */
/* lanes_per_atom (Tersoff, SW): lanes of one atom's group, 4, 8 or 16 (0 =
 * 8); a tile shape the autotuner picks per workload. */
typedef struct mbf_tersoff_tables {
    int ns;
    const double *tb;
    const double *tri;
    double r_cut;
} mbf_tersoff_tables;

int mbf_tersoff_eval(const mbf_system *sys, const mbf_nlist *nl,
                     const mbf_tersoff_tables *tab, const mbf_reduce_plan *plan,
                     int precision, int lanes_per_atom, void *workspace, size_t workspace_bytes,
                     double *forces, double *energy, double *virial, void *stream);

/* Tersoff adjoint for fitting: the vector-Jacobian product of (energy,
 * forces, virial) with respect to the tables, in float64.  Given upstream
 * gradients g_energy (n_struct), g_forces (n_atoms, 3) and g_virial
 * (n_struct, 9) -- any may be NULL for zero -- writes
 *   d_tb[e]  = sum_s gE_s dE_s/dtb[e] + sum_a gF_a . dF_a/dtb[e]
 *              + sum_s gW_s : dW_s/dtb[e]          (ns*ns, 10)
 * and d_tri likewise (ns^3, 8), for every table entry (the valid flag, m
 * and unused columns get 0).  Replaces the forward-difference Jacobian of
 * the reference's fit (fitting/driver.py:802-816 over
 * fitting/loss.py:263-319): one call instead of one loss evaluation per
 * parameter.  Zeta is recomputed per bond, nothing per triplet is stored;
 * the result is deterministic.  The workspace needs
 * mbf_tersoff_adjoint_workspace_bytes(n_slots, ns).                      */
size_t mbf_tersoff_adjoint_workspace_bytes(long long n_slots, int ns);
int mbf_tersoff_adjoint(const mbf_system *sys, const mbf_nlist *nl,
                        const mbf_tersoff_tables *tab, const double *g_energy,
                        const double *g_forces, const double *g_virial, void *workspace,
                        size_t workspace_bytes, double *d_tb, double *d_tri, void *stream);

/* ---- fit loss ----------------------------------------------------------
 * The reference's fit loss over a batch (fitting/loss.py:184-260, squared or
 * Huber, fitting/loss.py:29-48) and its gradient with respect to the
 * batch's energies, forces and virials -- the upstream gradients that
 * mbf_tersoff_adjoint / mbf_eam_adjoint take.  Structure s holds atoms
 * struct_off[s] .. struct_off[s+1]; its first n_orig[s] atoms are the
 * original cell's (the rest replicas of a thin cell, k_s = 1 / inv_k[s]
 * copies), with reference forces f_ref[fref_off[s] + a].  Per structure:
 *   e_sq = (E_s inv_k_s - n_s e_ref_s)^2
 *   f_sq = r0^2 sum_a |F_a - f_ref_a|^2 / (3 n_s)
 *   s_sq = (vol_s eps0)^2 mean_9 (W_s / vsup_s - s_ref_s)^2
 *   loss = sum_s cw_s [w_e h(e_sq) + fmask_s w_f h(f_sq) + smask_s w_s h(s_sq)]
 * h the identity (huber = 0) or sq -> 2 delta sqrt(sq) - delta^2 above
 * delta^2 (huber = 1, delta_e / delta_f / delta_s).  All pointers are device
 * arrays.  Sums run in a fixed order.                                    */
typedef struct mbf_fit_set {
    int n_struct, n_atoms;
    const int *struct_off;     /* (n_struct + 1) */
    const int *atom_struct;    /* (n_atoms,) */
    const int *n_orig;         /* (n_struct,) */
    const int *fref_off;       /* (n_struct,) first row of the structure in f_ref */
    const double *inv_k;       /* (n_struct,) 1 / replicas of the evaluated cell */
    const double *e_ref;       /* (n_struct,) reference energy per atom */
    const double *f_ref;       /* (sum n_orig, 3) */
    const double *s_ref;       /* (n_struct, 9) reference stress */
    const double *vol;         /* (n_struct,) volume of the original cell */
    const double *vsup;        /* (n_struct,) volume of the evaluated cell */
    const double *fmask;       /* (n_struct,) 1 if forces are fitted */
    const double *smask;       /* (n_struct,) 1 if stress is fitted */
    const double *cw;          /* (n_struct,) trust weight * scale^2 */
    double w_e, w_f, w_s, r0, eps0;
    int huber;
    double delta_e, delta_f, delta_s;
} mbf_fit_set;

size_t mbf_fit_loss_workspace_bytes(int n_struct);
/* Writes loss[0] and g_energy (n_struct), g_forces (n_atoms, 3), g_virial
 * (n_struct, 9), all device arrays; two launches on `stream`.            */
int mbf_fit_loss(const mbf_fit_set *set, const double *energy, const double *forces, const double *virial,
                 void *workspace, size_t workspace_bytes, double *loss, double *g_energy, double *g_forces,
                 double *g_virial, void *stream);

/* ---- Stillinger-Weber -------------------------------------------------
 * Replaces StillingerWeberPotential.compute (engine/stillinger_weber.py:
 * 900-1451), single- and multi-species.  tb (ns*ns, 8) rows [valid, eps,
 * sigma, a, A, B, p, q] of the two-body records; leg (ns*ns, 4) rows
 * [sigma, a, gamma, unused]; tri (ns*ns*ns, 4) rows [valid, eps*lambda/2,
 * costheta0, unused].  A single-species parameter dict is the ns = 1 case
 * with lambda halved over both neighbour orders.                         */
typedef struct mbf_sw_tables {
    int ns;
    const double *tb;
    const double *leg;
    const double *tri;
    double r_cut;
} mbf_sw_tables;

int mbf_sw_eval(const mbf_system *sys, const mbf_nlist *nl, const mbf_sw_tables *tab,
                const mbf_reduce_plan *plan, int precision, int lanes_per_atom, void *workspace,
                size_t workspace_bytes, double *forces, double *energy,
                double *virial, void *stream);

/* ---- measurement ------------------------------------------------------
 * Launch profiler: between begin and end every kernel launch of this library
 * is bracketed by CUDA events on its stream; end() synchronises the device
 * and writes "name launches total_ms" lines to buf.  Returns the number of
 * kernels listed.  No counterpart in the reference (its timing is
 * benchmarks/bench_force.py's wall clock).                                */
/* ---- site terms (heat flux) --------------------------------------------
 * mbf_*_eval_sites: the evaluation above plus the site-energy
 * decomposition of the reference's engine/site_terms.py:1-83 (Green-Kubo
 * heat flux, Fan et al. PRB 92, 094301): site_e (n_atoms) U_i, and per list
 * slot (centre i -> neighbour j) site_dudv (n_slots, 3) = dU_i/dv_ij and
 * site_vec (n_slots, 3) = v_ij (minimum image); slots beyond the cutoff get
 * dU/dv = 0.  Energy conventions per potential as the reference's
 * tersoff_site_terms (:312-437, U_i += fc (fR + b_ij fA) / 2 with the
 * centre's own bond order), sw_site_terms (:179-300, half the two-body term
 * plus the angles centred on i) and eam_site_terms (:440-479, F_i + half
 * the pair terms).  F_k = sum_m dUdv_m (delta_k,centre - delta_k,nbr)
 * rebuilds the forces.                                                    */
int mbf_tersoff_eval_sites(const mbf_system *sys, const mbf_nlist *nl,
                           const mbf_tersoff_tables *tab, const mbf_reduce_plan *plan,
                           int precision, int lanes_per_atom, void *workspace,
                           size_t workspace_bytes, double *forces, double *energy, double *virial,
                           double *site_e, double *site_dudv, double *site_vec, void *stream);
int mbf_sw_eval_sites(const mbf_system *sys, const mbf_nlist *nl, const mbf_sw_tables *tab,
                      const mbf_reduce_plan *plan, int precision, int lanes_per_atom,
                      void *workspace, size_t workspace_bytes, double *forces, double *energy,
                      double *virial, double *site_e, double *site_dudv, double *site_vec,
                      void *stream);
int mbf_eam_eval_sites(const mbf_system *sys, const mbf_nlist *nl, const mbf_eam_tables *tab,
                       const mbf_reduce_plan *plan, int precision, int lanes_per_atom,
                       void *workspace, size_t workspace_bytes, double *forces, double *energy,
                       double *virial, double *site_e, double *site_dudv, double *site_vec,
                       void *stream);

/* ---- velocity-Verlet NVE on the device ---------------------------------
 * The integrator of NVESimulation.run (solvers/molecular_dynamics.py:
 * 1969-2000) split around the force call: velocities in A/fs, masses in
 * amu, forces in eV/A, inv_mass[a] = EV_ANG_TO_AMU_ANG_FS2 / m_a.
 *
 * mbf_md_kick_drift: v += dt/2 * F * inv_mass; r += dt * v; then the wrap
 * of every position into its cell, frac = r @ inv(L), frac -= floor(frac),
 * frac >= 1 -> 0, r = frac @ L (positions updated in place: `positions`
 * is the mbf_system's array).                                            */
int mbf_md_kick_drift(const mbf_system *sys, double *positions, double *velocities,
                      const double *forces, const double *inv_mass, double dt, void *stream);

/* v += dt/2 * F * inv_mass, and the kinetic energy of every structure,
 * 1/2 sum m v^2 / EV_ANG_TO_AMU_ANG_FS2 in eV (_kinetic_energy,
 * solvers/molecular_dynamics.py:239-244; m v^2 / conv = v^2 / inv_mass),
 * summed in a fixed order: partial (mbf_md_partial_count(n_atoms) doubles
 * per structure) is scratch, and the pair (potential energy energy[s],
 * kinetic energy) is written to thermo at row (*counter) mod thermo_rows
 * (thermo: (thermo_rows, n_struct, 2)); *counter (device) then advances
 * by one.  One launch: *done (device word) must be 0 and is left at 0.  */
int mbf_md_partial_count(int n_atoms);
int mbf_md_kick(const mbf_system *sys, double *velocities, const double *forces,
                const double *inv_mass, double dt, const double *energy,
                double *partial, double *thermo, int thermo_rows, int *counter, unsigned *done,
                void *stream);

/* mbf_md_kick_drift and mbf_md_skin_check (below, with a graph condition
 * handle or 0 and no status word) in one launch: the displacement maxima
 * d_max (n_struct device words) and *done must be 0 and are left at 0;
 * the other arguments are mbf_md_skin_check's.                           */
int mbf_md_kick_drift_check(const mbf_system *sys, double *positions, double *velocities,
                            const double *forces, const double *inv_mass, double dt,
                            const double *ref_positions, double r_list, double r_cut,
                            unsigned long long *d_max, unsigned *done, double *d_log, int rows,
                            int *counter, int *gate, unsigned long long cond_handle, void *stream);

/* mbf_md_kick of one step followed by mbf_md_kick_drift_check of the
 * next, in one launch (both half kicks use the forces of the step that
 * ended; every stored value, the thermo row and the decision equal those of
 * the two launches).  thermo_counter / skin_counter are the two entries'
 * counters; d_max (n_struct device words) and *done must be 0 and are left
 * at 0.                                                                   */
int mbf_md_kick_kick_drift_check(const mbf_system *sys, double *positions, double *velocities,
                                 const double *forces, const double *inv_mass, double dt,
                                 const double *energy, double *partial, double *thermo,
                                 int thermo_rows, int *thermo_counter, const double *ref_positions,
                                 double r_list, double r_cut, unsigned long long *d_max,
                                 double *d_log, int rows, int *skin_counter, int *gate,
                                 unsigned long long cond_handle, unsigned *done, void *stream);

/* The reference's rebuild decision (engine/neighborlist.py:613-673 with
 * the lattice fixed: rebuild iff r_list - 2 d <= r_cut, d = max_a |MIC(r_a -
 * r_ref_a)| since the last rebuild) evaluated on the device every step:
 * records d at row (*counter) mod rows of d_log (rows, n_struct), advances
 * *counter, and writes the decision (1 = rebuild) to *gate (device int).
 * cond_handle (from mbf_capture_cond_create, or 0) is set to the decision,
 * gating an IF branch that holds mbf_nl_rebuild_async and
 * mbf_md_rebuild_done.  A non-null status gets MBF_STATUS_SKIN when the
 * decision is 1 (fixed-interval runs, where it is an assertion).        */
int mbf_md_skin_check(const mbf_system *sys, const double *ref_positions, double r_list,
                      double r_cut, double *d_scratch, double *d_log, int rows, int *counter,
                      int *gate, int *status, unsigned long long cond_handle, void *stream);

/* After a rebuild: ref_positions = positions, ++*rebuild_count (device). */
int mbf_md_rebuild_done(const mbf_system *sys, double *ref_positions, int *rebuild_count,
                        void *stream);

/* Conditional branches inside a stream capture (CUDA graph IF nodes), so a
 * captured MD step rebuilds its list only when the device decides to.
 * mbf_capture_cond_create: a handle on the graph `stream` is capturing
 * (value 0 at each launch).  mbf_capture_if_begin: adds an IF node on that
 * handle after the stream's current work, makes it the stream's only
 * dependency, and starts capturing `body_stream` (another stream) into the
 * branch; mbf_capture_if_end ends the branch. No counterpart in the
 * reference. */
int mbf_capture_cond_create(void *stream, unsigned long long *cond_handle);
int mbf_capture_if_begin(void *stream, void *body_stream, unsigned long long cond_handle);
int mbf_capture_if_end(void *body_stream);

void mbf_profile_begin(void);
int mbf_profile_end(char *buf, size_t cap);

/* Sustained FMA throughput (FLOP/s, 2 per FMA) of the current GPU in
 * float64 (precision 0) or float32 (1): the compute roofline denominator.
 * scratch >= 148 * 8 * 256 * 8 bytes of device memory. */
int mbf_peak_probe(int precision, void *scratch, size_t scratch_bytes, double *flops,
                   void *stream);

#ifdef __cplusplus
}
#endif

#endif /* MBFORCE_H */
