/*
 * libsemisim_b200 - C ABI of the B200 solve path of SemiSim 3D.
 *
 * The library is a drop-in for the reference core semiconductor_3d.c: it exports every
 * api3_* entry point with the reference's exact C signature and semantics (one global
 * device; 1 = ok / 0 = failure; getters NaN for a bad index or no solution), so the
 * reference's main.py, its sweeps and validate.py load it unchanged through
 *     SEMISIM_SO=<path>/libsemisim_b200.so
 * (semibuild.py:516-522).  Each declaration names the reference function it replaces
 * (semiconductor_3d.c:<line>) and, where one exists, the ctypes binding that loads it.
 *
 * The solve path (prepare, equilibrium, Newton-Poisson, Scharfetter-Gummel continuity,
 * Gummel / Anderson, continuation, terminal currents) runs on the GPU; set-up calls only
 * record the device and work without one.  Every physics model of the reference runs
 * there too, on tensor and on general (prism / graph, api3_set_mesh_graph) meshes: gate
 * tunnelling, thermionic-emission metal contacts, impact and incomplete ionisation, MLDA
 * quantum confinement, Lombardi surface mobility with the 4H-SiC Coulomb term and deep
 * traps.  The standalone model evaluators (api3_tun_eval, api3_mlda_factor,
 * api3_lombardi, api3_coulomb_inv) run on the host and return the reference's values.
 * Without a CUDA device the solve entries return 0 with a message on stderr; there is no
 * CPU solve path.
 */
#ifndef SEMISIM_B200_H
#define SEMISIM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* replaces semiconductor_3d.c:4570; bound at main.py:176 */
void api3_init(void);
/* replaces semiconductor_3d.c:4599; bound at main.py:3498 */
void api3_set_threads(int n);
/* replaces semiconductor_3d.c:4607 */
void api3_set_verbose(int v);
/* replaces semiconductor_3d.c:4618; bound at main.py:3509 */
int api3_trap_species(int type, int ref, double E, double sn, double sp);
/* replaces semiconductor_3d.c:4629; bound at main.py:3510 */
int api3_trap_add(int sid, int n, const int *nodes, const double *dens);
/* replaces semiconductor_3d.c:4645 */
void api3_traps_clear(void);
/* replaces semiconductor_3d.c:4646; bound at main.py:3511 */
int api3_charge_add(int n, const int *nodes, const double *rho);
/* replaces semiconductor_3d.c:4653 */
int api3_n_trap_entries(void);
/* replaces semiconductor_3d.c:4657; bound at main.py:187 */
void api3_set_models(int flags);
/* replaces semiconductor_3d.c:4660; bound at main.py:188 */
void api3_set_caxis(int ax);
/* replaces semiconductor_3d.c:4661 */
int api3_get_caxis(void);
/* replaces semiconductor_3d.c:4663; bound at main.py:177 */
int api3_add_material(int id, double T);
/* replaces semiconductor_3d.c:4671; bound at main.py:3512 */
int api3_set_mat_tau(int mi, double tn, double tp);
/* replaces semiconductor_3d.c:4679; bound at main.py:179 */
int api3_set_grid_coords(int Nx,int Ny,int Nz,const double *xs,const double *ys,const double *zs);
/* replaces semiconductor_3d.c:4693; bound at main.py:178 */
void api3_set_grid(int Nx,int Ny,int Nz,double Lx,double Ly,double Lz);
/* replaces semiconductor_3d.c:4708; bound at main.py:180 */
void api3_set_solver(int mp,int mc,int mg,double tp,double tc,double op,double oc);
/* replaces semiconductor_3d.c:4718; bound at main.py:181 */
void api3_set_region(int x0,int y0,int z0,int x1,int y1,int z1,int midx,double Nd,double Na);
/* replaces semiconductor_3d.c:4731 */
void api3_add_fixed_charge(int x0,int y0,int z0,int x1,int y1,int z1,double Nf);
/* replaces semiconductor_3d.c:4742; bound at main.py:186 */
void api3_add_sheet_charge(int axis,int idx,int a0,int a1,int b0,int b1,double sigma);
/* replaces semiconductor_3d.c:4757; bound at main.py:184 */
int api3_add_contact_ex(int face,int i0,int i1,int j0,int j1,int k0,int k1, int bc,double V,double pm,double tox,double Nox);
/* replaces semiconductor_3d.c:4772; bound at main.py:182 */
void api3_add_contact(int face,int i0,int i1,int j0,int j1,int bc,double V,double pm);
/* replaces semiconductor_3d.c:4775; bound at main.py:185 */
void api3_clear_contacts(void);
/* replaces semiconductor_3d.c:4779; bound at main.py:3500 */
int api3_set_gate_stack(int cid,int nl,const int *mat,const double *t);
/* replaces semiconductor_3d.c:4795; bound at main.py:3503 */
int api3_set_mesh_graph(int N,int E,const int *rp,const int *cj,const double *h, const double *ar,const double *vol,const double *pos);
/* replaces semiconductor_3d.c:4806; bound at main.py:3504 */
int api3_is_graph(void);
/* replaces semiconductor_3d.c:4808; bound at main.py:3505 */
void api3_set_node_data(const int *mat,const double *Nd,const double *Na,const double *Nf);
/* replaces semiconductor_3d.c:4821; bound at main.py:3506 */
int api3_set_con_nodes(int cid,int n,const int *nodes,const double *areas);
/* replaces semiconductor_3d.c:4838; bound at main.py:3507 */
void api3_set_walls(const double *w);
/* replaces semiconductor_3d.c:4844; bound at main.py:3501 */
int api3_get_ntp(int cid);
/* replaces semiconductor_3d.c:4855; bound at validate.py:42 */
double api3_tun_eval(int smat,int nl,const int *mat,const double *t,double psi, double phin,double phip,double Vg,double pm,double *out);
/* replaces semiconductor_3d.c:4869; bound at validate.py:43 */
double api3_mlda_factor(int mi,double a,double b,int hole);
/* replaces semiconductor_3d.c:4878; bound at validate.py:46 */
double api3_coulomb_inv(int mi,double F,double n,double NC,double NA);
/* replaces semiconductor_3d.c:4885 */
int api3_set_surface_mobility(int mi,double delta,double eta,double mu1);
/* replaces semiconductor_3d.c:4894; bound at validate.py:44 */
double api3_lombardi(int mi,double mub,double F,double Nt,double Dw,int hole);
/* replaces semiconductor_3d.c:4898; bound at main.py:191 */
void api3_set_contact_V(int cid,double V);
/* replaces semiconductor_3d.c:4899; bound at main.py:3449 */
int api3_get_ncon(void);
/* replaces semiconductor_3d.c:4900; bound at main.py:192 */
double api3_get_contact_I(int cid);
/* replaces semiconductor_3d.c:4901; bound at main.py:193 */
double api3_get_contact_A(int cid);
/* replaces semiconductor_3d.c:4902; bound at main.py:194 */
double api3_get_contact_In(int cid);
/* replaces semiconductor_3d.c:4904; bound at main.py:195 */
double api3_get_contact_Ifloor(int cid);
/* replaces semiconductor_3d.c:4906; bound at main.py:196 */
double api3_get_contact_Iraw(int cid);
/* replaces semiconductor_3d.c:4907; bound at main.py:3499 */
int api3_get_aa_depth(void);
/* replaces semiconductor_3d.c:4908; bound at main.py:3497 */
double api3_get_contact_Vsolved(int cid);
/* replaces semiconductor_3d.c:4922; bound at main.py:3494 */
void api3_request_stop(void);
/* replaces semiconductor_3d.c:4923; bound at main.py:3495 */
void api3_clear_stop(void);
/* replaces semiconductor_3d.c:4924 */
int api3_stop_requested(void);
/* replaces semiconductor_3d.c:4926; bound at main.py:3496 */
void api3_get_progress(double *out);
/* replaces semiconductor_3d.c:4928; bound at main.py:189 */
int api3_solve(void);
/* replaces semiconductor_3d.c:4930; bound at main.py:190 */
int api3_resolve(void);
/* replaces semiconductor_3d.c:4934; bound at main.py:215 */
void api3_iv_sweep(int cid,double Vs,double Ve,int Npts,double *Varr,double *Jarr,int *Carr);
/* replaces semiconductor_3d.c:4958; bound at main.py:217 */
void api3_iv_sweep2(int cid,double Vs,double Ve,int Npts,double *Varr, double *Iarr,double *Farr,int *Carr);
/* replaces semiconductor_3d.c:4981; bound at main.py:204 */
double api3_get_Emax(void);
/* replaces semiconductor_3d.c:5003; bound at main.py:198 */
int api3_get_Nx(void);
/* replaces semiconductor_3d.c:5004; bound at main.py:198 */
int api3_get_Ny(void);
/* replaces semiconductor_3d.c:5005; bound at main.py:198 */
int api3_get_Nz(void);
/* replaces semiconductor_3d.c:5006; bound at main.py:199 */
int api3_get_conv(void);
/* replaces semiconductor_3d.c:5007; bound at main.py:199 */
int api3_get_iter(void);
/* replaces semiconductor_3d.c:5008; bound at main.py:199 */
double api3_get_res(void);
/* replaces semiconductor_3d.c:5009; bound at main.py:200 */
double api3_get_xs(int i);
/* replaces semiconductor_3d.c:5010; bound at main.py:200 */
double api3_get_ys(int j);
/* replaces semiconductor_3d.c:5011; bound at main.py:200 */
double api3_get_zs(int l);
/* replaces semiconductor_3d.c:5012; bound at validate.py:41 */
double api3_get_Cref(void);
/* replaces semiconductor_3d.c:5013; bound at main.py:197 */
long long api3_get_stat(int w);
/* replaces semiconductor_3d.c:5019; bound at validate.py:45 */
void api3_set_predictor(int on);
/* replaces semiconductor_3d.c:5023; bound at main.py:3999 */
int api3_get_state(double *phi, double *phin, double *phip);
/* replaces semiconductor_3d.c:5030; bound at main.py:4000 */
int api3_set_state(const double *phi, const double *phin, const double *phip);
/* replaces semiconductor_3d.c:5043 */
double api3_get_time(int w);
/* replaces semiconductor_3d.c:5048; bound at main.py:201 */
double api3_mat_ni(int mi);
/* replaces semiconductor_3d.c:5049; bound at main.py:201 */
double api3_mat_Eg(int mi);
/* replaces semiconductor_3d.c:5127; bound at main.py:202 */
void api3_bulk_copy(int which,double *out);
/* replaces semiconductor_3d.c:5137; bound at main.py:3513 */
void api3_carrier_sums(double *out);
/* replaces semiconductor_3d.c:5192; bound at main.py:208 */
int api3_charge_partition(const int *cterm);
/* replaces semiconductor_3d.c:5248; bound at main.py:209 */
int api3_terminal_charges(int nt, double *Qt);
/* replaces semiconductor_3d.c:5284; bound at main.py:212 */
int api3_face_J(int ax, int carrier, double *out);
/* replaces semiconductor_3d.c:5300; bound at main.py:210 */
int api3_charge_owner(int *out);
/* replaces semiconductor_3d.c:5308; bound at main.py:211 */
double api3_ins_field_max(double *pos);
/* replaces semiconductor_3d.c:5341; bound at validate.py:1229 */
double api3_get_phi(int k);
/* replaces semiconductor_3d.c:5342 */
double api3_get_n(int k);
/* replaces semiconductor_3d.c:5343 */
double api3_get_p(int k);
/* replaces semiconductor_3d.c:5344 */
double api3_get_Ec(int k);
/* replaces semiconductor_3d.c:5345 */
double api3_get_Ev(int k);
/* replaces semiconductor_3d.c:5346 */
double api3_get_Efn(int k);
/* replaces semiconductor_3d.c:5347 */
double api3_get_Efp(int k);
/* replaces semiconductor_3d.c:5348 */
double api3_get_Jx(int k);
/* replaces semiconductor_3d.c:5349 */
double api3_get_Jy(int k);
/* replaces semiconductor_3d.c:5350 */
double api3_get_Jz(int k);
/* replaces semiconductor_3d.c:5351 */
double api3_get_mun(int k);
/* replaces semiconductor_3d.c:5352 */
double api3_get_mup(int k);
/* replaces semiconductor_3d.c:5353 */
double api3_get_R(int k);

/* ---- additive entries (no counterpart in the reference) ---- */

/* Pin the low-field mobility of material mi to constants mun / mup (m^2/Vs),
   independent of doping and temperature; 1 = done, 0 = bad index or value.  The oracle
   harness exports the same entry so both libraries are set up identically. */
int api3_set_mat_mobility(int mi, double mun, double mup);

/* More solver instances.  The reference core has one global device; here every
   api3_* call acts on the calling thread's current instance (instance 0 = the global
   device of the reference ABI).  Independent devices solved from different host
   threads run concurrently on the GPU, each instance on its own CUDA stream.
   api3b_new: a new, empty instance; returns its handle (>= 1).
   api3b_use: make instance h current for the calling thread (0: the global one);
              1 = done, 0 = no such instance.
   api3b_current: the calling thread's current instance.
   api3b_free: release an instance and its device memory; 1 = done. */
int api3b_new(void);
int api3b_use(int h);
int api3b_current(void);
int api3b_free(int h);

/* No counterpart in the reference (its solves are FP64 only).  Linear-solve precision of
   the current instance, kept across api3_init:
     0  FP64 throughout (the reference's arithmetic);
     1  refined: the Krylov iterations and the multigrid hierarchy of every linear solve run
        in FP32 (FP32 copy of the operator, FP32 vectors, dot products summed in FP64)
        inside FP64 iterative refinement: x and r = b - A x stay FP64 with the FP64
        operator, and the solve stops on the reference's FP64 rule.  Continuity solves
        (BiCGSTAB) refine explicitly; the Newton-Poisson corrections (PCG) are refined by
        the Newton loop's FP64 residual (PCG tolerances below 1e-5 stay FP64).  A refinement
        that stops gaining hands the solve to the FP64 solver;
    -1  the library default (SEMISIM_B200_PRECISION=mixed at api3_init selects 1, else 0).
   api3b_set_precision returns the previous setting; api3b_get_precision the mode in
   effect (0 or 1). */
int api3b_set_precision(int mode);
int api3b_get_precision(void);

/* No counterpart in the reference.  Persistent linear solves (library-wide): with mode 1
   (the default; SEMISIM_B200_PERSIST=0 switches it off) every multigrid-preconditioned
   PCG / BiCGSTAB solve of an instance runs as one cooperative kernel launch - all its
   iterations, V-cycles and FP64 refinement steps, with grid-wide barriers between the
   dependent passes; mode 0 launches one kernel per pass inside device-looped CUDA graphs.
   Both stop on the same rules.  `blocks` caps the blocks of one launch (0: every SM's
   worth; SEMISIM_B200_PBLOCKS sets it at start-up), so that instances solved concurrently
   from several host threads can share the GPU.  -1 leaves a value unchanged.  Returns the
   previous mode. */
int api3b_set_persist(int mode, int blocks);

/* No counterpart in the reference.  Grid share of the current instance's persistent solves:
   blocks > 0 caps each of its launches at that many blocks (below the library-wide cap of
   api3b_set_persist), 0 removes the share, -1 only reads it.  Instances solved at the same
   time from several host threads run side by side when their shares add up to at most
   the GPU's co-resident blocks (one per SM); otherwise their cooperative launches take
   turns.  A share changes only the launch shape, never the stop rules; the grid
   reductions' order follows the block count, so results are reproducible per share.
   The share belongs to the instance and survives api3_init.  Returns the previous share. */
int api3b_set_share(int blocks);

/* No counterpart in the reference.  Order of the sweep predictor (library-wide): 1 (the
   default; the reference's secant step x1 + s (x1 - x0) from the last two sweep points) or 2
   (quadratic: the Lagrange polynomial through the last three sweep points' solutions,
   evaluated at the new bias; used when the three biases and the new one lie on one line,
   else the secant step).  It only sets the Gummel loop's starting point; the stop rules are
   the same.  SEMISIM_B200_PRED_ORDER sets it at api3_init.  Other values only read it.
   Returns the previous order. */
int api3b_set_pred_order(int order);

/* No counterpart in the reference (it has no learned component).  Learned sweep predictor
   of the current instance: a per-node MLP (48 features -> 3 x 128 SiLU -> 3, BF16 weights,
   FP32 accumulation) corrects the sweep predictor's linear extrapolation
   x1 + s (x1 - x0) of (psi, phi_n, phi_p) at the first continuation step of a new bias
   point.  It only changes the Gummel loop's starting point: the loop still stops on the
   same tolerances, and a seeded step that fails is redone from the linear guess.
     api3b_seed_set_model: load api3b_seed_nparam() FP32 parameters (W1 [128][48], b1 [128],
        W2 [128][128], b2, W3 [128][128], b3, W4 [8][128] with rows 3-7 zero, b4 [8]) into the
        instance (after its first solve) and enable the seed; 1 = done, 0 = wrong size /
        no device memory yet.
     api3b_seed_enable: 1 on, 0 off (linear guess only); returns the previous setting.
        api3_init switches the seed off (the model stays loaded for api3b_seed_enable(1)).
     api3b_seed_stats: seeded predictor steps and seeded steps redone from the linear guess. */
int api3b_seed_set_model(const float *params, int n);
int api3b_seed_enable(int on);
void api3b_seed_stats(long long *used, long long *fallbacks);
int api3b_seed_nparam(void);

/* No counterpart in the reference.  Launch-shape autotuner of the current instance: rows
   per block of the row-blocked multigrid passes, blocks of the grid-stride node kernels,
   and the level size where the small-level kernel takes over, chosen by timing V-cycles of
   the instance's own hierarchy (in the precision its solves use) on the GPU.
     mode 0: default shapes; 1: tune now; 2: reuse the shapes cached for this mesh shape
     and precision, tuning when there are none.  Call after the instance's first solve,
     with no other GPU work of the process running.  Returns the chosen V-cycle time in
     microseconds (0 for mode 0, -1 before the first solve or on a general (graph) mesh,
     whose multigrid has no tunable shapes).
   api3b_tune_get: the shapes in use (zcap: most row blocks per pass; may be null); returns
   1 when they came from the tuner. */
double api3b_autotune(int mode);

/* No counterpart in the reference (its callers that multiply solves - main.py's cap_matrix
   C-V perturbations, main.py:4034-4087, and solve_floating's secant, main.py:3575-3636 -
   restore a state and call api3_resolve once per bias vector).  Solves n bias vectors V
   (n x ncon volts) from the current instance's solved state, each independently, on up to
   `workers` worker instances at once (<= 0: min(n, 8)), each with its own device memory,
   CUDA stream and host thread.  Outputs per vector: terminal currents I (n x ncon), floors
   Iflr and converged flags conv (both may be null).  The current instance is unchanged.
   Returns the number of converged solves, -1 without a solution or on a device error.
   api3b_resolve_batch_free releases the current instance's workers (they are kept for
   later calls; api3b_free releases the freed instance's workers too). */
int api3b_resolve_batch(int n, const double *V, double *I, double *Iflr, int *conv, int workers);
int api3b_resolve_batch_free(void);
int api3b_tune_get(int *rpb, int *grid_cap, int *small_nodes, int *zcap);

/* No counterpart in the reference.  For callers that cannot allocate device memory
   (their memory belongs to another allocator, or a cudaMalloc / cudaFree on their path is
   not acceptable): r = b - A x for a 7-point stencil A (7 arrays of N = Nx*Ny*Nz doubles:
   diagonal, x-, x+, y-, y+, z-, z+), norms[0] = ||r||_2 and norms[1] = the BiCGSTAB
   rounding floor sqrt(sum_a (sum_b |A_ab x_b| + |b_a|)^2).  A7, x, b, r: the caller's
   device buffers on one GPU (each checked; a host buffer, a buffer on another GPU or an r
   that overlaps A7, x or b is refused before any launch); norms: host.  The calling
   thread's current device is restored on return.  Allocates nothing: its reduction scratch is a
   fixed ~38 KB device array that every GPU loading the library holds until exit.  At most
   2^30 nodes (larger sizes are refused with a message).  The first call on a GPU looks up
   that array (cudaGetSymbolAddress): make it before any stream capture.  Calls share the
   array and use the default stream; calls that overlap on one GPU race.  1 = done. */
int api3b_stencil_residual_noalloc(const double *A7, const double *x, const double *b, int Nx, int Ny, int Nz,
                                   double *r, double *norms);

#ifdef __cplusplus
}
#endif
#endif /* SEMISIM_B200_H */
