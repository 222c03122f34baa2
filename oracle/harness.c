/*
 * Oracle harness (test infrastructure only).
 *
 * This translation unit #includes the reference core semiconductor_3d.c from the
 * reference checkout (-I<reference>), unmodified, so that its static kernels and the
 * global device `gdev` (semiconductor_3d.c:366) become reachable.  It adds:
 *
 *   - api3_set_mat_mobility: an additive entry that pins a material's low-field
 *     mobility to a constant (the reference has Masetti / Arora only,
 *     semiconductor_3d.c:646-662).  The B200 library exports the same symbol, so one
 *     driver sets up both sides identically.
 *   - hx_* dump hooks that run one reference kernel on the prepared device and copy
 *     its outputs into caller buffers.  They are the golden-vector source for the
 *     kernel-level parity tests.
 *
 * Nothing here is shipped or timed.  Built by oracle/Makefile into oracle/_ref/.
 */
#include "semiconductor_3d.c"

/* ---- additive entry: constant low-field mobility (m^2/Vs) of material mi.
   mob_low (semiconductor_3d.c:646-662) returns mu_min + (mu_max-mu_min)/(...),
   which is the constant when mu_min == mu_max and the temperature exponents are 0. */
int api3_set_mat_mobility(int mi, double mun, double mup){
    if(mi<0 || mi>=gdev.n_mats || !(mun>0.) || !(mup>0.)) return 0;
    Mat *m=&gdev.mats[mi];
    m->mas_on=0;
    m->mu_n_min=m->mu_n_max=mun; m->mu_p_min=m->mu_p_max=mup;
    m->mt_min=m->mt_max_n=m->mt_max_p=0.;
    mark_changed(&gdev);
    return 1;
}

long hx_N(void){ return gdev.allocated ? (long)NN(&gdev) : 0; }
int  hx_prepare(void){ return prepare(&gdev); }
int  hx_equilibrium(void){ if(!prepare(&gdev)) return 0; return equilibrium(&gdev); }
int  hx_nlev(void){ return gdev.nlev; }
double hx_cref(void){ return gdev.Cref; }

/* per-node masks after prepare (semiconductor_3d.c:1638-1775) */
void hx_masks(int *kind, int *con, int *gate){
    size_t N=NN(&gdev);
    for(size_t k=0;k<N;k++){ kind[k]=gdev.kind[k]; con[k]=gdev.con_mask[k]; gate[k]=gdev.gate_mask[k]; }
}
int hx_rob(long *k, double *A, int *c){
    for(int r=0;r<gdev.n_rob;r++){ if(k) k[r]=(long)gdev.rob_k[r]; if(A) A[r]=gdev.rob_A[r]; if(c) c[r]=gdev.rob_c[r]; }
    return gdev.n_rob;
}
void hx_contact_area(double *A){ for(int c=0;c<gdev.n_cons;c++) A[c]=gdev.cons[c].A; }
/* contact record: V, phi_m, tox, qox, bc, face */
int hx_contact(int c, double *out){
    if(c<0||c>=gdev.n_cons) return 0;
    const Con *cn=&gdev.cons[c];
    out[0]=cn->V; out[1]=cn->phi_m; out[2]=cn->tox; out[3]=cn->qox; out[4]=cn->bc; out[5]=cn->face;
    return 1;
}

static double *hx_arr(int which){
    Dev *d=&gdev;
    switch(which){
    case 0: return d->phi; case 1: return d->phi_n; case 2: return d->phi_p;
    case 3: return d->n; case 4: return d->p; case 5: return d->mu_n; case 6: return d->mu_p;
    case 7: return d->bgn; case 8: return d->eps; case 9: return d->Nd; case 10: return d->Na;
    case 11: return d->Nf;
    }
    return NULL;
}
/* which: 0 phi, 1 phi_n, 2 phi_p, 3 n, 4 p, 5 mu_n, 6 mu_p, 7 bgn, 8 eps, 9 Nd, 10 Na, 11 Nf;
   16..21: face mobility fmu[0..5] (semiconductor_3d.c:256) */
int hx_get(int which, double *out){
    size_t N=NN(&gdev);
    if(which>=16 && which<22){                   /* tensor meshes only (a graph keeps edge mobilities) */
        if(gdev.unstr) return 0;
        for(size_t k=0;k<N;k++) out[k]=(double)gdev.fmu[which-16][k];
        return 1;
    }
    double *a=hx_arr(which); if(!a) return 0;
    memcpy(out,a,N*sizeof(double)); return 1;
}
int hx_set(int which, const double *in){
    size_t N=NN(&gdev);
    if(which>=16 && which<22){
        if(gdev.unstr) return 0;
        for(size_t k=0;k<N;k++) gdev.fmu[which-16][k]=(mu_t)in[k];
        return 1;
    }
    double *a=hx_arr(which); if(!a) return 0;
    memcpy(a,in,N*sizeof(double)); return 1;
}

static void hx_Va(double *Va){ for(int c=0;c<gdev.n_cons;c++) Va[c]=gdev.cons[c].V; }
static void hx_dump_sten(const Sten *A, size_t N, double *A7){
    if(!A7) return;
    const double *src[7]={A->c,A->xm,A->xp,A->ym,A->yp,A->zm,A->zp};
    for(int q=0;q<7;q++) memcpy(A7+(size_t)q*N,src[q],N*sizeof(double));
}

/* poisson_eval (semiconductor_3d.c:2732-2789) at the given psi and the contact
   voltages now set; returns ||F/diag|| */
double hx_poisson_eval(const double *phi, int build, double *F, double *A7, double *sc){
    double Va[NC_MAX]; hx_Va(Va);
    size_t N=NN(&gdev);
    double *Fw=malloc(N*sizeof(double));
    double r=poisson_eval(&gdev,phi,Va,build,Fw);
    if(F) memcpy(F,Fw,N*sizeof(double));
    if(build){ hx_dump_sten(&gdev.A,N,A7); if(sc) memcpy(sc,gdev.sc,N*sizeof(double)); }
    free(Fw);
    return r;
}
void hx_apply_bc(void){ double Va[NC_MAX]; hx_Va(Va); set_vrange(&gdev,Va); apply_bc(&gdev,Va); }
void hx_rebuild_np(void){ rebuild_np(&gdev); }
void hx_mob0_init(void){ mob0_init(&gdev); }
/* the edge mobilities of either mesh (upd_mob, semiconductor_3d.c:3007-3008 dispatch) */
void hx_upd_mob(void){
    if(gdev.unstr) upd_mob_ref_g(&gdev,gdev.phi_n,gdev.phi_p);
    else upd_mob_ref(&gdev,gdev.phi_n,gdev.phi_p);
}
void hx_clamp_qf(void){ clamp_qf(&gdev); }
double hx_vlo(void){ return gdev.vlo; }
double hx_vhi(void){ return gdev.vhi; }

/* cont_assemble (semiconductor_3d.c:3067-3106) */
void hx_cont_assemble(int hole, double *A7, double *rhs, double *sc, double *dsc){
    size_t N=NN(&gdev);
    memset(gdev.tk,0,N*sizeof(double)); memset(gdev.tg,0,N*sizeof(double)); memset(gdev.gii,0,N*sizeof(double));
    cont_assemble(&gdev,hole);
    hx_dump_sten(&gdev.A,N,A7);
    if(rhs) memcpy(rhs,gdev.rhs,N*sizeof(double));
    if(sc) memcpy(sc,gdev.sc,N*sizeof(double));
    if(dsc) memcpy(dsc,gdev.dsc,N*sizeof(double));
}
/* cont_update (semiconductor_3d.c:3112-3146) after hx_cont_assemble of the same carrier */
double hx_cont_update(int hole, const double *sol, double lo, double hi, double *dq){
    size_t N=NN(&gdev);
    memcpy(gdev.sol,sol,N*sizeof(double));
    return cont_update(&gdev,hole,dq,lo,hi);
}
/* float_fix (semiconductor_3d.c:3159-3228) on sol, after hx_cont_assemble; sol is rescaled in place */
int hx_float_fix(int hole, double *sol){
    size_t N=NN(&gdev);
    memcpy(gdev.sol,sol,N*sizeof(double));
    int r=float_fix(&gdev,hole);
    memcpy(sol,gdev.sol,N*sizeof(double));
    return r;
}
/* terminal_currents (semiconductor_3d.c:3598-3623) */
void hx_terminal_currents(double *I, double *S, double *In){
    double Iw[NC_MAX],Sw[NC_MAX];
    terminal_currents(&gdev,Iw,Sw);
    for(int c=0;c<gdev.n_cons;c++){ I[c]=Iw[c]; S[c]=Sw[c]; if(In) In[c]=gdev.cons[c].In; }
}
/* one solve of the continuity equation with the reference's own BiCGSTAB + MG
   (semiconductor_3d.c:3580-3594); returns the weighted max |dq| */
double hx_solve_cont(int hole, double *dq){
    double Va[NC_MAX]; hx_Va(Va); set_vrange(&gdev,Va);
    double dm=0.;
    solve_cont(&gdev,hole,dq,gdev.vlo,gdev.vhi,&dm);
    return dm;
}
/* neutral_psi (semiconductor_3d.c:1787-1804) */
double hx_neutral_psi(long k, double V){ return neutral_psi(&gdev,(size_t)k,V); }

/* ---- multigrid hierarchy (semiconductor_3d.c:1894-2148) on the matrix now in gdev.A.
   qsign 0: Poisson (plain aggregation); +1/-1 continuity with the level-0 weights dsc. */
int hx_mg_setup(int qsign){
    gdev.mg_qsign=qsign; gdev.mg_w = qsign ? gdev.dsc : NULL;
    mg_setup(&gdev);
    return gdev.nlev;
}
/* dims: Nx,Ny,Nz,cx,cy,cz of level L; A7, pw, ph, ilu may be NULL */
int hx_mg_level(int L, int *dims, double *A7, double *pw, double *ph){
    if(L<0||L>=gdev.nlev) return 0;
    const Lev *v=&gdev.lev[L];
    if(dims){ dims[0]=v->Nx; dims[1]=v->Ny; dims[2]=v->Nz; dims[3]=v->cx; dims[4]=v->cy; dims[5]=v->cz; }
    hx_dump_sten(&v->A,v->N,A7);
    if(pw && v->pw) memcpy(pw,v->pw,v->N*sizeof(double));
    if(ph && v->ph) memcpy(ph,v->ph,v->N*sizeof(double));
    return 1;
}
/* level-L operators: y = A x (level L), restriction to L+1, prolongation from L+1 */
int hx_mg_matvec(int L, const double *x, double *y){
    if(L<0||L>=gdev.nlev) return 0;
    matvec_L(&gdev,&gdev.lev[L],x,NULL,y); return 1;
}
int hx_mg_restrict(int L, const double *r, double *bc){
    if(L<0||L>=gdev.nlev-1) return 0;
    restrict_sum(&gdev.lev[L],&gdev.lev[L+1],r,bc, L==0 ? gdev.mg_w : NULL); return 1;
}
int hx_mg_prolong(int L, const double *xc, double *x){
    if(L<0||L>=gdev.nlev-1) return 0;
    prolong_add(&gdev.lev[L],&gdev.lev[L+1],xc,x); return 1;
}
/* coarsest dense solve (semiconductor_3d.c:2050-2081) */
int hx_mg_coarse_solve(const double *b, double *x){
    dense_solve(&gdev.lev[gdev.nlev-1],b,x); return 1;
}
/* BiCGSTAB rounding floor sqrt(sum (sum_b |A_ab x_b| + |b_a|)^2) of the level-0
   matrix (semiconductor_3d.c:2244-2268) */
double hx_bicg_floor(const double *b, const double *x){
    const Lev *v0=&gdev.lev[0]; const Sten *A=&v0->A;
    const int Nx=v0->Nx,Ny=v0->Ny,Nz=v0->Nz; const size_t NxNy=(size_t)Nx*Ny; double fl=0.;
    for(int l=0;l<Nz;l++) for(int j=0;j<Ny;j++){
        size_t k=IDX(0,j,l,Nx,Ny);
        for(int i=0;i<Nx;i++,k++){
            double s=fabs(A->c[k]*x[k])+fabs(b[k]);
            if(i>0)    s+=fabs(A->xm[k]*x[k-1]);
            if(i<Nx-1) s+=fabs(A->xp[k]*x[k+1]);
            if(j>0)    s+=fabs(A->ym[k]*x[k-Nx]);
            if(j<Ny-1) s+=fabs(A->yp[k]*x[k+Nx]);
            if(l>0)    s+=fabs(A->zm[k]*x[k-NxNy]);
            if(l<Nz-1) s+=fabs(A->zp[k]*x[k+NxNy]);
            fl+=s*s;
        }
    }
    return sqrt(fl);
}

/* incomplete-ionisation constants of the prepared device (ION_W per node), 0 when every
   dopant is ionised */
int hx_ion(double *out){
    if(!gdev.ion) return 0;
    if(out) memcpy(out,gdev.ion,ION_W*NN(&gdev)*sizeof(double));
    return ION_W;
}

/* metal contacts: te_update at the contacts' stage voltages, and the entry / column
   records (counts in cnt[2] = n_te, n_tc; arrays may be NULL) */
void hx_te_update(void){
    double Va[NC_MAX];
    for(int c=0;c<gdev.n_cons;c++) Va[c]=gdev.cons[c].V;
    te_update(&gdev,Va);
}
/* gate tunnelling: tun_update at the contacts' stage voltages, and the path / column
   records (counts in cnt[2] = n_tp, n_col; arrays may be NULL) */
void hx_tun_update(void){
    double Va[NC_MAX];
    for(int c=0;c<gdev.n_cons;c++) Va[c]=gdev.cons[c].V;
    tun_update(&gdev,Va);
}
int hx_tun(int *cnt, double *tpG, double *colK, long *tpk, long *colk){
    cnt[0]=gdev.n_tp; cnt[1]=gdev.n_col;
    if(tpG) memcpy(tpG,gdev.tp_G,2*gdev.n_tp*sizeof(double));
    if(colK) memcpy(colK,gdev.col_K,2*gdev.n_col*sizeof(double));
    if(tpk) for(int p=0;p<gdev.n_tp;p++) tpk[p]=(long)gdev.tp_k[p];
    if(colk) for(int q=0;q<gdev.n_col;q++) colk[q]=(long)gdev.col_k[q];
    return gdev.n_tp;
}
/* install an image-force band (qcn, qcp; N each) as te_update would have left it */
void hx_set_qc(const double *qcn, const double *qcp){
    size_t N=NN(&gdev);
    memcpy(gdev.qcn,qcn,N*sizeof(double)); memcpy(gdev.qcp,qcp,N*sizeof(double));
    if(gdev.imgn) memcpy(gdev.imgn,qcn,N*sizeof(double));
    if(gdev.imgp) memcpy(gdev.imgp,qcp,N*sizeof(double));
}
int hx_te(int *cnt, double *teK, double *teG, double *tcK, double *tcG, double *tcI, double *qcn, double *qcp){
    cnt[0]=gdev.n_te; cnt[1]=gdev.n_tc;
    if(teK) memcpy(teK,gdev.te_K,2*gdev.n_te*sizeof(double));
    if(teG) memcpy(teG,gdev.te_G,2*gdev.n_te*sizeof(double));
    if(tcK) memcpy(tcK,gdev.tc_K,2*gdev.n_tc*sizeof(double));
    if(tcG) memcpy(tcG,gdev.tc_G,2*gdev.n_tc*sizeof(double));
    if(tcI) memcpy(tcI,gdev.tc_I,2*gdev.n_tc*sizeof(double));
    if(qcn) memcpy(qcn,gdev.qcn,NN(&gdev)*sizeof(double));
    if(qcp) memcpy(qcp,gdev.qcp,NN(&gdev)*sizeof(double));
    return gdev.n_te;
}

/* ---- scalar physics (semiconductor_3d.c:646-697) */
double hx_B(double x){ return B(x); }
double hx_mob_low(int mi, double N, int hole){ return mob_low(&gdev.mats[mi],N,hole); }
double hx_mob_hf(double mu0, double E, double vsat, double beta){ return mob_hf(mu0,E,vsat,beta); }
void hx_recomb(int mi, double ni, double tf, double n, double p, double *out){
    recomb(&gdev.mats[mi],ni,tf,n,p,&out[0],&out[1],&out[2]);
}
/* material record as plain doubles (order of hx_mat_fields below) */
int hx_mat(int mi, double *out){
    if(mi<0||mi>=gdev.n_mats) return 0;
    mat_prepare(&gdev);
    const Mat *m=&gdev.mats[mi];
    double v[]={m->T,m->VT,m->Eg,m->chi,m->eps_r,m->Nc,m->Nv,m->ni,
                m->mu_n_max,m->mu_p_max,m->mu_n_min,m->mu_p_min,m->Nref_n,m->Nref_p,m->alpha_n,m->alpha_p,
                m->mt_min,m->mt_max_n,m->mt_max_p,m->mt_Nref,m->mt_alpha,(double)m->mas_on,
                m->vsat_n,m->vsat_p,m->beta_n,m->beta_p,m->tau_n0,m->tau_p0,m->Cn,m->Cp,m->Brad,m->tau_Nref,
                m->bgn_E,m->bgn_N,m->bgn_C,m->lnc,m->lnv,(double)m->insulator,m->ani_n,m->ani_p,
                (double)m->ion_on,m->ion_w[0],m->ion_w[1],m->ion_Ed[0],m->ion_Ed[1],m->ion_ad[0],m->ion_ad[1],
                m->ion_gd,m->ion_Ea,m->ion_aa,m->ion_ga,
                (double)m->ii_on,m->ii_a[0][0],m->ii_a[0][1],m->ii_a[1][0],m->ii_a[1][1],
                m->ii_b[0][0],m->ii_b[0][1],m->ii_b[1][0],m->ii_b[1][1],m->ii_E0[0],m->ii_E0[1],
                m->ii_m[0],m->ii_m[1],m->ii_g};
    memcpy(out,v,sizeof v);
    return (int)(sizeof v/sizeof v[0]);
}

/* graph multigrid hierarchy built by api3_set_mesh_graph (gmg_alloc,
   semiconductor_3d.c:2475-2512): level L's node count and pattern size, and when the
   buffers are given its CSR pattern and (below the coarsest) every node's aggregate.
   Returns the number of levels (0 without a graph device). */
int hx_gmg_level(int L, int *n_out, int *nnz_out, int *rp, int *cj, int *agg){
    if(!gdev.allocated || !gdev.unstr) return 0;
    int nl=gdev.nlev;
    if(L<0 || L>=nl) return nl;
    const Lev *v=&gdev.lev[L];
    int n=(int)v->N;
    if(n_out) *n_out=n;
    if(nnz_out) *nnz_out=v->rp[n];
    if(rp) for(int i=0;i<=n;i++) rp[i]=v->rp[i];
    if(cj) for(int e=0;e<v->rp[n];e++) cj[e]=v->cj[e];
    if(agg && L<nl-1 && v->agg) for(int i=0;i<n;i++) agg[i]=v->agg[i];
    return nl;
}

/* the graph of a general-mesh device (api3_set_mesh_graph, semiconductor_3d.c:981-1041):
   CSR rp (N + 1), cj, undirected edge id ue, lengths h and dual areas ar (E each), node
   volumes (N); null buffers are skipped.  Returns E (0 without a graph device). */
int hx_graph(int *rp, int *cj, int *ue, double *h, double *ar, double *vol){
    if(!gdev.allocated || !gdev.unstr) return 0;
    size_t N=NN(&gdev); int E=gdev.nE;
    if(rp) for(size_t k=0;k<=N;k++) rp[k]=gdev.grp[k];
    if(cj) memcpy(cj,gdev.gcol,(size_t)E*sizeof(int));
    if(ue) memcpy(ue,gdev.gue,(size_t)E*sizeof(int));
    if(h) memcpy(h,gdev.gh,(size_t)E*8);
    if(ar) memcpy(ar,gdev.ga,(size_t)E*8);
    if(vol) memcpy(vol,gdev.gvol,N*8);
    return E;
}
/* the off-diagonals of the last assembled graph system (poisson_core_g / cont_assemble_g,
   semiconductor_3d.c:4181-4217, 4314-4351), per directed edge; returns E */
int hx_graph_vals(double *gval){
    if(!gdev.allocated || !gdev.unstr) return 0;
    if(gval) memcpy(gval,gdev.gval,(size_t)gdev.nE*8);
    return gdev.nE;
}
/* edge mobilities of the graph (upd_mob_ref_g, semiconductor_3d.c:4241-4293) per undirected
   edge; returns their number */
int hx_graph_mob(double *mun, double *mup){
    if(!gdev.allocated || !gdev.unstr) return 0;
    for(int e=0;e<gdev.nUE;e++){ if(mun) mun[e]=(double)gdev.gmu[0][e]; if(mup) mup[e]=(double)gdev.gmu[1][e]; }
    return gdev.nUE;
}

/* the values of graph multigrid level L after hx_mg_setup (g_galerkin, semiconductor_3d.c:
   2575-2594): off-diagonals in the level's CSR order (nnz) and the diagonal (N); returns nnz */
int hx_gmg_vals(int L, double *va, double *dg){
    if(!gdev.allocated || !gdev.unstr || L<0 || L>=gdev.nlev) return -1;
    const Lev *v=&gdev.lev[L];
    int n=(int)v->N, nnz=v->rp[n];
    if(va) memcpy(va,v->va,(size_t)nnz*8);
    if(dg) memcpy(dg,v->dg,(size_t)n*8);
    return nnz;
}

/* impact-ionisation pair generation of every node at the present state (ii_update,
   semiconductor_3d.c:4486-4523), 1/s per control volume; returns 1 */
int hx_ii_update(double *gii){
    ii_update(&gdev);
    if(gii) memcpy(gii,gdev.gii,NN(&gdev)*sizeof(double));
    return 1;
}
