/*
 * libsemisim_b200 - kernel-level test and measurement hooks (b200x_*).
 *
 * Not part of the reference ABI (no counterpart in semiconductor_3d.c).  They run one
 * device kernel of the solve path on the calling thread's current instance, with inputs
 * and outputs through host buffers, so the parity tests can compare every kernel with
 * the oracle on seeded states, and bench.py can time kernels with CUDA events.
 */
#ifndef SEMISIM_B200_TESTING_H
#define SEMISIM_B200_TESTING_H

#ifdef __cplusplus
extern "C" {
#endif

/* prepare the recorded device on the GPU (masks, Robin areas, materials); 1 = done */
int b200x_prepare(void);
/* per node: kind, contact id + 1, gate id + 1, Robin area (m^2) */
int b200x_masks(int *kind, int *con, int *gate, double *robA);
/* the incomplete-ionisation constants of the prepared device, 4 per node (two donor
   sites, the acceptor, the neutral majority density); returns 4, or 0 when every dopant
   is fully ionised (semiconductor_3d.c:1472-1510) */
int b200x_ion(double *out);
/* metal contacts (models bit 6): te_update at the contacts' voltages (returns 0 without
   metal contacts), and the entry / column records: cnt[0] entries, cnt[1] column nodes;
   emission terms te_K / te_G (2 per entry), column exchange terms tc_K / tc_G and
   image-force lowering tc_I (2 per column node), per-node band lowering qcn / qcp (N);
   null arrays are skipped (semiconductor_3d.c:3390-3571) */
int b200x_te_update(void);
int b200x_set_qc(const double *qcn, const double *qcp);   /* install an image-force band (N each) */
/* gate tunnelling (models bit 5): tun_update at the contacts' voltages (0 without paths), and
   the records: cnt[0] paths, cnt[1] column nodes; injection tp_G (2 per path), escape rates
   col_K (2 per column node), path and column node indices; null arrays are skipped
   (semiconductor_3d.c:3326-3371) */
int b200x_tun_update(void);
int b200x_tun(int *cnt, double *tpG, double *colK, long long *tpk, long long *colk);
/* graph multigrid hierarchy of a CSR graph, host only (replaces reading the reference's
   gdev.lev[] after gmg_alloc, semiconductor_3d.c:2475-2512): level L's size, pattern and
   aggregates; returns the number of levels */
int b200x_gmg_plan(int N, const int *rp, const int *cj, const double *h, const double *ar, int L,
                   int *n_out, int *nnz_out, int *rp_out, int *cj_out, int *agg_out);
/* graph multigrid set-up on the system now assembled (qsign 0 Poisson, +-1 continuity) and
   level L's couplings in CSR order and diagonal (replaces reading gdev.lev[L].va / dg after
   gmg_setup, semiconductor_3d.c:2643-2653); returns the coupling count */
int b200x_gmg_vals(int qsign, int L, double *va, double *dg);
int b200x_te(int *cnt, double *teK, double *teG, double *tcK, double *tcG, double *tcI, double *qcn, double *qcp);
/* device state arrays: 0 psi, 1 phi_n, 2 phi_p, 3 n, 4 p, 5/6 low-field mobility n/p,
   7 sol, 8 rhs, 9 sc, 10 dsc, 16..21 face mobility (n x,y,z; p x,y,z), 22..24 sweep history
   h1 (psi, phi_n, phi_p now), 25..27 e2 (one step back) */
int b200x_set(int which, const double *in);
int b200x_get(int which, double *out);
double b200x_vlo(void);
double b200x_vhi(void);
void b200x_apply_bc(void);
void b200x_rebuild_np(void);
/* charge-neutral start state at the present contact voltages (no Newton solve) */
void b200x_init_state(void);
void b200x_upd_mob(void);
void b200x_clamp_qf(void);
/* Poisson residual, Jacobian (7 x N) and sc at psi; returns ||F/diag|| */
double b200x_poisson(const double *phi, double *F, double *A7, double *sc);
/* scaled SG continuity system of carrier `hole` at the present state */
void b200x_cont_assemble(int hole, double *A7, double *rhs, double *sc, double *dsc);
/* carrier / quasi-Fermi update from sol; returns the weighted max |dq| */
double b200x_cont_update(int hole, const double *sol, double lo, double hi, double *dq);
/* terminal currents, scales and electron parts per contact */
void b200x_currents(double *I, double *S, double *In);
/* multigrid hierarchy of the system now in A (qsign 0 Poisson, +1/-1 continuity) */
int b200x_mg_setup(int qsign);
int b200x_mg_level(int L, int *dims, double *A7, double *pw);
/* Krylov solves of the system now in A / rhs */
int b200x_bicgstab(int maxit, double rtol, double atol, int qsign, const double *x0, double *sol, double *rn,
                   double *r0);
int b200x_pcg(int maxit, double rtol, double *sol);
/* The persistent solves' bounded barrier wait, exercised: a cooperative launch of nb
   blocks on the current instance's barrier record whose last block never arrives.
   Returns the error word (1 when the others gave up after wait_s seconds) and in
   *gave_up how many blocks reported it (nb - 1); -1 if the launch failed. */
int b200x_persist_probe(int nb, double wait_s, int *gave_up);
/* Barrier timeline of the next persistent solve (measurement hook): n > 0 arms a timeline of
   n barriers (returns 0); n == 0 copies it to out - per barrier the first and the last
   block's arrival and the release as block 0 saw it (globaltimer ns) - disarms it and
   returns 1 when a launch filled it, with that launch's blocks in *blocks. */
int b200x_persist_trace(int n, unsigned long long *out, int *blocks);
/* Block cap of the persistent solves that the calling host thread launches (measurement
   hook): n > 0 caps the grid at n blocks, 0 removes the cap, n < 0 only reads it.  Returns
   the previous cap. */
int b200x_persist_tblocks(int n);
/* floating-block balance of a continuity solution (in place) */
int b200x_float_fix(int hole, double *sol);
/* learned predictor on the present history arrays (22-24 h1, 25-27 e2 of b200x_set /
   b200x_get): psi, phi_n, phi_p = h1 + s (h1 - e2) + VT * MLP; 1 = done */
int b200x_seed_run(double s, const double *dv4);
/* thermal voltage of the reference material (0 before prepare) */
double b200x_vtref(void);
/* refinement steps and FP64 take-overs of the instance's refined continuity solves */
void b200x_ir_stats(long long *steps, long long *fallbacks);
/* device memory of the instance (bytes) */
long long b200x_device_bytes(void);
/* CUDA device of the solver (before its first solve); 1 = done */
int b200x_set_device(int dev);
/* microseconds per launch of one kernel over `reps` back-to-back launches (0-10 FP64
   linear algebra, 11-16 the FP32 twins and the FP64 refinement update, 20 continuity
   assembly, 21 Poisson build) */
double b200x_bench(int which, int reps);
/* CUDA-event timer on the instance's stream: op 0 start, op 1 stop -> elapsed ms */
double b200x_stream_timer(int op);
/* launch accounting and per-kernel-class event timing */
int b200x_prof(int on);
int b200x_prof_read(int id, double *ms, double *count, double *bytes);
const char *b200x_prof_name(int id);
int b200x_prof_detail(int q, int *id, double *nodes, double *ms, double *count);
unsigned long long b200x_launches(void);

#ifdef __cplusplus
}
#endif
#endif /* SEMISIM_B200_TESTING_H */
