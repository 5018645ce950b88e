/*
 * fm_oracle.c -- CPU FP64 restatement of Flowmol's per-timestep MD hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA path in
 * flowmol_b200/ is compared against.  It is linked only by tests/, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg; the product
 * library never calls it.
 *
 * Parity status: the reference (Fortran 90 + MPI) cannot be compiled in this
 * environment (no gfortran, no MPI) and ships no golden force / pair-list
 * vectors.  The geometry rules below are pinned against the values the
 * reference printed into runs/Intrinsic_Interface/results/simulation_header;
 * the restart format is pinned against src/reorder_restart/read_final_state.py
 * run on runs/Intrinsic_Interface/initial_state.  Pair lists, forces, the
 * integrator and the rebuild criterion are restated line by line from the
 * Fortran cited at each function, but for those parts parity is UNPINNED by
 * reference outputs (only analytic known-answer cases pin them).
 *
 * Numerics follow the reference build (gfortran -O3 -funroll-loops on x86-64,
 * no -march, hence no FMA contraction): compile with -ffp-contract=off and
 * without -ffast-math.  Array layout mirrors the Fortran modules: r, v, a are
 * column-major (3, cap) so r[3*n+k] is r(k+1, n+1).  Molecule numbers inside
 * the linked lists are 1-based like the reference; halo images occupy
 * np+1 .. np+halo_np.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_OK 0
#define ORC_ERR_ALLOC 1
#define ORC_ERR_ESCAPE 2
#define ORC_ERR_FEWCELLS 3
#define ORC_ERR_BOND 4
#define ORC_ERR_PARAM 5

typedef struct orc {
    /* ---- parameters (modules.f90 computational/physical constants) ---- */
    int np, halo_np, cap, globalnp;
    double domain[3], halfdomain[3], cellsidelength[3];
    int ncells[3];
    double rcutoff, rcutoff2, rneighbr2, delta_rneighbr[3], delta_t, potshift;
    double density, potential_sLRC, pressure_sLRC;
    int tplot, teval, iter;
    int force_list;        /* 0 all pairs, 2 full list, 3 half list */
    int rebuild_criteria;  /* 0 vmax, 1 fixed, 2 displacement */
    int fixed_rebuild;
    int integration_algorithm; /* 0 leap-frog, 1 velocity Verlet */
    int potential_flag;    /* 0 LJ, 1 FENE polymer */
    double k_c, R_0;
    int solvent_flag;      /* 1: Soddemann solvent (chainID 0 = solvent molecule) */
    double sod_eps[3];     /* well depth by chain beads in the pair: eps_ss, eps_ps, eps_pp */
    int max_funcy;
    /* ---- state (arrays_MD) ---- */
    double *r, *v, *a;        /* (3, cap) */
    int *glob_no;             /* cap: identity carried to halo images */
    int *halo_src;            /* cap: source molecule (1-based) of an image */
    signed char *halo_shift;  /* (3, cap): -1/0/+1 domain shift of an image */
    double *potenergymol, *virialmol, *potenergymol_POLY;
    double *rdisp;            /* (3, np) displacement criterion */
    /* polymer connectivity: chain/subchain/funcy/bin_bflag per molecule, bond(max_funcy, cap) */
    int *chainID, *subchainID, *funcy;
    int *bflag;               /* (4, cap) bin_bflag words */
    int *bond;                /* (max_funcy, np) 1-based molecule numbers, 0 = empty */
    int *bondcount;           /* np */
    /* ---- cell linked lists (linklist.f90 cellinfo/node) ---- */
    int ncell_tot;
    int *cellnp, *cellhead;   /* (nc+2)^3 */
    int *cn_molno, *cn_next;  /* node pool */
    int cn_count, cn_cap;
    /* ---- neighbour lists (linklist.f90 neighbrinfo) ---- */
    int *Nlist, *nhead;       /* np */
    int *nn_molno, *nn_next;
    long nn_count, nn_cap;
    /* ---- checkrebuild / record ---- */
    double rmax, simtime;
    /* tag_move (ensemble 6) data: molecular_properties.f90 */
    int ensemble;             /* 0 NVE, 6 tag_move */
    int *tag;                 /* cap */
    double *rtether, *slidev; /* (3, cap) */
    double teth_k2, teth_k4, teth_k6;
    int nthermo;
    double therm_T[2], zeta[2];
    /* virial pressure tensor (pressure_outflag 1) */
    int pressure_outflag;
    double *rfmol;            /* (9, cap) */
    double Pxy[9];
    int nstress;
    /* Mie_potential 1: moltype (cap, 1-based) and the lookup tables of
     * setup_mie_potential, (i,j) at [(i-1) + MIET*(j-1)] */
    int mie;
    int *moltype;
    double mie_mass[16], mie_eps[256], mie_lr[256], mie_la[256], mie_C[256], mie_alpha[256], mie_shift[256],
        mie_k[256], mie_r0[256];
    /* angular_potential: angular_k_lookup / angular_r0_lookup (ntypes^3,
     * (i,j,k) at [(i-1) + ang_nt*((j-1) + ang_nt*(k-1))]) */
    int angular, ang_nt;
    double *ang_k, *ang_t0;
    double vsum, mv2sum, potenergysum, virial;
    double kinenergy, potenergy, totenergy, temperature, pressure;
    int rebuild_count;
} orc;

/* ------------------------------------------------------------------------ */
/* setup_set_parameters.f90                                                  */
/* ------------------------------------------------------------------------ */

/* set_parameters_global_domain, initial_config_flag 0
 * (setup_set_parameters.f90:1545-1580): L_i = n_i / (density/4)**(1/nd). */
void orc_global_domain(const int nunits[3], double density, double domain_out[3],
                       double unitsize_out[3], double *volume_out)
{
    double vol = 1.0;
    for (int k = 0; k < 3; k++) {
        domain_out[k] = (double)nunits[k] / pow(density / 4.0, 1.0 / 3.0);
        vol = vol * domain_out[k];
    }
    for (int k = 0; k < 3; k++) unitsize_out[k] = domain_out[k] / (double)nunits[k];
    *volume_out = vol;
}

/* Soddemann solvent constants (polymer_info_MD, modules.f90:456-462).  sod_a,
 * sod_b and wca_cut2 are default-real literals in the reference, so their
 * FP64 values are the single-precision roundings: (double)(float)literal. */
#define SOD_CUT 1.5
#define SOD_CUT2 2.25
static double sod_a(void) { return (double)3.1730728678f; }
static double sod_b(void) { return (double)-0.85622864544f; }
static double wca_cut2(void) { return (double)1.25992104989487f; }

/* set_parameters_cells (setup_set_parameters.f90:1848-1903).  solvent_flag
 * 1 (Soddemann) raises rcutoff to sod_cut when rneighbr is below it and
 * leaves rneighbr2 (1871-1876); *rcutoff_io is rcutoff in and after.
 * Returns ORC_ERR_FEWCELLS where the reference aborts (fewer than 3 cells). */
int orc_set_parameters_cells(const double domain[3], double *rcutoff_io, const double delta[3],
                             int potential_flag, int solvent_flag, double R_0, int ncells_out[3],
                             double cellside_out[3], double *rneighbr2_out)
{
    double rcutoff = *rcutoff_io;
    double rneighbr = rcutoff + (delta[0] + delta[1] + delta[2]) / 3.0;
    double rneighbr2 = rneighbr * rneighbr;
    if (potential_flag == 1 && solvent_flag == 0 && rneighbr < R_0) { /* FENE override, 1865-1869 */
        rneighbr = R_0;
        rneighbr2 = R_0 * R_0;
    }
    if (potential_flag == 1 && solvent_flag == 1 && rneighbr < SOD_CUT) rcutoff = SOD_CUT;
    *rcutoff_io = rcutoff;
    for (int k = 0; k < 3; k++) ncells_out[k] = (int)floor(domain[k] / (rcutoff + delta[k]));
    *rneighbr2_out = rneighbr2;
    if (ncells_out[0] < 3 || ncells_out[1] < 3 || ncells_out[2] < 3) return ORC_ERR_FEWCELLS;
    for (int k = 0; k < 3; k++) cellside_out[k] = domain[k] / (double)ncells_out[k];
    return ORC_OK;
}

/* Integer powers as gfortran -O3 expands x**n (repeated multiplication). */
static inline double p3(double s) { return s * s * s; }
static inline double p6(double s) { double t = p3(s); return t * t; }
static inline double p12(double s) { double t = p6(s); return t * t; }

/* LJ_accijmag / LJ_energy (setup_set_parameters.f90:105-135). */
static inline double lj_accijmag(double s)
{
    double s2 = s * s, s4 = s2 * s2, s7 = s4 * s2 * s;
    return 48.0 * (s7 - 0.5 * s4);
}
static inline double lj_energy(double s, double potshift)
{
    return 4.0 * (p6(s) - p3(s)) - potshift;
}

double orc_lj_accijmag(double invrij2) { return lj_accijmag(invrij2); }
double orc_lj_energy(double invrij2, double potshift) { return lj_energy(invrij2, potshift); }
/* potshift = 4(rc^-12 - rc^-6) (setup_set_parameters.f90:1222) */
double orc_potshift(double rcutoff)
{
    return 4.0 * (1.0 / p12(rcutoff) - 1.0 / p6(rcutoff));
}

/* FENE_accijmag / FENE_energy (setup_set_parameters.f90:348-380). */
static inline double fene_accijmag(double rij2, double k_c, double R_0)
{
    return -k_c / (1.0 - (rij2 / (R_0 * R_0)));
}
static inline double fene_energy(double rij2, double k_c, double R_0)
{
    return 0.5 * k_c * R_0 * R_0 * log(1.0 - (rij2 / (R_0 * R_0)));
}

/* Mie_potential 1 (setup_set_parameters.f90:149-204, 384-437): constants by
 * the types of the two molecules (a halo image has its source's type, as
 * messenger_updateborders sends it, messenger.MPI.f90:693,764). */
#define MIET 16
static inline int type_of(const orc *s, int n) /* 1-based molecule or image */
{
    return n <= s->np ? s->moltype[n - 1] : s->moltype[s->halo_src[n - 1] - 1];
}
static inline double mass_of(const orc *s, int n) /* LJ_mass / Mie_mass */
{
    return s->mie ? s->mie_mass[type_of(s, n) - 1] : 1.0;
}
static inline double pair_accijmag(const orc *s, double invrij2, int i, int j)
{
    if (!s->mie) return lj_accijmag(invrij2);
    int q = (type_of(s, i) - 1) + MIET * (type_of(s, j) - 1);
    double C = s->mie_C[q], eps = s->mie_eps[q], lr = s->mie_lr[q], la = s->mie_la[q], al = s->mie_alpha[q];
    return C * eps * (lr * pow(invrij2, 0.5 * lr + 1) - al * la * pow(invrij2, 0.5 * la + 1));
}
static inline double pair_energy(const orc *s, double invrij2, int i, int j)
{
    if (!s->mie) return lj_energy(invrij2, s->potshift);
    int q = (type_of(s, i) - 1) + MIET * (type_of(s, j) - 1);
    double C = s->mie_C[q], eps = s->mie_eps[q], lr = s->mie_lr[q], la = s->mie_la[q], al = s->mie_alpha[q];
    return C * eps * (pow(invrij2, 0.5 * lr) - al * pow(invrij2, 0.5 * la)) - s->mie_shift[q];
}
static inline double harmonic_accijmag(const orc *s, double rij2, int i, int j)
{
    int q = (type_of(s, i) - 1) + MIET * (type_of(s, j) - 1);
    double rm = sqrt(rij2);
    return -s->mie_k[q] * (rm - s->mie_r0[q]) / rm;
}
static inline double harmonic_energy(const orc *s, double rij2, int i, int j)
{
    int q = (type_of(s, i) - 1) + MIET * (type_of(s, j) - 1);
    double d = sqrt(rij2) - s->mie_r0[q];
    return 0.5 * s->mie_k[q] * (d * d);
}

/* ------------------------------------------------------------------------ */
/* allocation                                                                */
/* ------------------------------------------------------------------------ */

static void *xcalloc(size_t n, size_t sz) { return calloc(n ? n : 1, sz); }

void orc_free(orc *s);

/* Creates a state for np molecules.  extralloc mirrors
 * set_parameters_allocate (setup_set_parameters.f90:1248-1290): room for the
 * halo images behind the real molecules. */
orc *orc_create(int np, const double domain[3], double rcutoff, const double delta[3],
                double delta_t, int tplot, int force_list, int potential_flag,
                double k_c, double R_0, int rebuild_criteria, int fixed_rebuild,
                double density, int sLRC_flag, int *err)
{
    orc *s = (orc *)xcalloc(1, sizeof(orc));
    *err = ORC_OK;
    if (!s) { *err = ORC_ERR_ALLOC; return NULL; }
    s->np = np; s->globalnp = np;
    for (int k = 0; k < 3; k++) {
        s->domain[k] = domain[k];
        s->halfdomain[k] = 0.5 * domain[k];
        s->delta_rneighbr[k] = delta[k];
    }
    s->rcutoff = rcutoff;
    s->rcutoff2 = rcutoff * rcutoff;
    s->delta_t = delta_t;
    s->tplot = tplot;
    s->teval = tplot;
    s->force_list = force_list;
    s->potential_flag = potential_flag;
    s->k_c = k_c; s->R_0 = R_0;
    s->max_funcy = 4;
    s->rebuild_criteria = rebuild_criteria;
    s->fixed_rebuild = fixed_rebuild > 0 ? fixed_rebuild : 1;
    s->integration_algorithm = 1;
    s->density = density;
    s->potshift = orc_potshift(rcutoff);
    if (sLRC_flag) {
        const double pi = 3.14159265358979323846;
        s->potential_sLRC = 8.0 * pi * density * (1.0 / (9.0 * pow(rcutoff, 9)) - 1.0 / (3.0 * p3(rcutoff)));
        s->pressure_sLRC = 8.0 * pi * (density * density) *
                           (4.0 / (9.0 * pow(rcutoff, 9)) - 2.0 / (3.0 * p3(rcutoff)));
    }
    double rc_cells = rcutoff;
    int rc = orc_set_parameters_cells(s->domain, &rc_cells, delta, potential_flag, 0, R_0,
                                      s->ncells, s->cellsidelength, &s->rneighbr2);
    if (rc != ORC_OK && force_list != 0) { *err = rc; orc_free(s); return NULL; }
    if (rc != ORC_OK) { s->ncells[0] = s->ncells[1] = s->ncells[2] = 1; }
    /* halo capacity: every boundary molecule may be imaged up to 7 times */
    s->cap = np * 8 + 1024;
    size_t cap = (size_t)s->cap;
    s->r = (double *)xcalloc(3 * cap, sizeof(double));
    s->v = (double *)xcalloc(3 * cap, sizeof(double));
    s->a = (double *)xcalloc(3 * cap, sizeof(double));
    s->glob_no = (int *)xcalloc(cap, sizeof(int));
    s->halo_src = (int *)xcalloc(cap, sizeof(int));
    s->halo_shift = (signed char *)xcalloc(3 * cap, 1);
    s->potenergymol = (double *)xcalloc(cap, sizeof(double));
    s->potenergymol_POLY = (double *)xcalloc(cap, sizeof(double));
    s->virialmol = (double *)xcalloc(cap, sizeof(double));
    s->chainID = (int *)xcalloc(cap, sizeof(int));
    s->subchainID = (int *)xcalloc(cap, sizeof(int));
    s->funcy = (int *)xcalloc(cap, sizeof(int));
    s->bflag = (int *)xcalloc(4 * cap, sizeof(int));
    s->bond = (int *)xcalloc((size_t)s->max_funcy * (size_t)np, sizeof(int));
    s->bondcount = (int *)xcalloc((size_t)np, sizeof(int));
    s->tag = (int *)xcalloc(cap, sizeof(int));
    s->rtether = (double *)xcalloc(3 * cap, sizeof(double));
    s->slidev = (double *)xcalloc(3 * cap, sizeof(double));
    s->rfmol = (double *)xcalloc(9 * cap, sizeof(double));
    s->ncell_tot = (s->ncells[0] + 2) * (s->ncells[1] + 2) * (s->ncells[2] + 2);
    s->cellnp = (int *)xcalloc((size_t)s->ncell_tot, sizeof(int));
    s->cellhead = (int *)xcalloc((size_t)s->ncell_tot, sizeof(int));
    s->cn_cap = s->cap;
    s->cn_molno = (int *)xcalloc(cap, sizeof(int));
    s->cn_next = (int *)xcalloc(cap, sizeof(int));
    s->Nlist = (int *)xcalloc((size_t)np, sizeof(int));
    s->nhead = (int *)xcalloc((size_t)np, sizeof(int));
    s->nn_cap = (long)np * 16 + 1024;
    s->nn_molno = (int *)xcalloc((size_t)s->nn_cap, sizeof(int));
    s->nn_next = (int *)xcalloc((size_t)s->nn_cap, sizeof(int));
    for (int n = 0; n < np; n++) s->glob_no[n] = n + 1;
    if (!s->r || !s->v || !s->a || !s->nn_molno || !s->nn_next || !s->cn_molno) {
        *err = ORC_ERR_ALLOC; orc_free(s); return NULL;
    }
    return s;
}

void orc_free(orc *s)
{
    if (!s) return;
    free(s->r); free(s->v); free(s->a); free(s->glob_no); free(s->halo_src); free(s->halo_shift);
    free(s->potenergymol); free(s->potenergymol_POLY); free(s->virialmol); free(s->rdisp);
    free(s->chainID); free(s->subchainID); free(s->funcy); free(s->bflag); free(s->bond);
    free(s->bondcount);
    free(s->tag); free(s->rtether); free(s->slidev); free(s->rfmol); free(s->moltype);
    free(s->ang_k); free(s->ang_t0);
    free(s->cellnp); free(s->cellhead); free(s->cn_molno); free(s->cn_next);
    free(s->Nlist); free(s->nhead); free(s->nn_molno); free(s->nn_next);
    free(s);
}

/* SOLVENT_INFO (setup_read_input.f90:275-296): solvent_flag and the well
 * depths, then the geometry again as set_parameters_cells derives it with the
 * flag (setup_set_parameters.f90:1848-1903); potshift and the long-range
 * corrections follow the raised rcutoff (:1222-1238).  Call before setup. */
int orc_set_solvent(orc *s, int solvent_flag, double eps_pp, double eps_ps, double eps_ss)
{
    if (solvent_flag != 0 && solvent_flag != 1) return ORC_ERR_PARAM;
    if (solvent_flag == 1 && (s->potential_flag != 1 || s->force_list != 3)) return ORC_ERR_PARAM;
    s->solvent_flag = solvent_flag;
    s->sod_eps[0] = eps_ss; s->sod_eps[1] = eps_ps; s->sod_eps[2] = eps_pp;
    double rc = s->rcutoff;
    int ncells[3];
    double cs[3], rn2;
    int rc_err = orc_set_parameters_cells(s->domain, &rc, s->delta_rneighbr, s->potential_flag, solvent_flag,
                                          s->R_0, ncells, cs, &rn2);
    if (rc_err) return rc_err;
    s->rcutoff = rc;
    s->rcutoff2 = rc * rc;
    s->rneighbr2 = rn2;
    s->potshift = orc_potshift(rc);
    if (s->potential_sLRC != 0.0 || s->pressure_sLRC != 0.0) {
        const double pi = 3.14159265358979323846;
        s->potential_sLRC = 8.0 * pi * s->density * (1.0 / (9.0 * pow(rc, 9)) - 1.0 / (3.0 * p3(rc)));
        s->pressure_sLRC = 8.0 * pi * (s->density * s->density) * (4.0 / (9.0 * pow(rc, 9)) - 2.0 / (3.0 * p3(rc)));
    }
    for (int k = 0; k < 3; k++) { s->ncells[k] = ncells[k]; s->cellsidelength[k] = cs[k]; }
    int nt = (ncells[0] + 2) * (ncells[1] + 2) * (ncells[2] + 2);
    if (nt != s->ncell_tot) {
        int *np_ = (int *)xcalloc((size_t)nt, sizeof(int)), *hd = (int *)xcalloc((size_t)nt, sizeof(int));
        if (!np_ || !hd) { free(np_); free(hd); return ORC_ERR_ALLOC; }
        free(s->cellnp); free(s->cellhead);
        s->cellnp = np_; s->cellhead = hd;
        s->ncell_tot = nt;
    }
    return ORC_OK;
}

/* Accessors used by the ctypes wrapper. */
double *orc_r(orc *s) { return s->r; }
double *orc_v(orc *s) { return s->v; }
double *orc_a(orc *s) { return s->a; }
int *orc_glob_no(orc *s) { return s->glob_no; }
double *orc_potenergymol(orc *s) { return s->potenergymol; }
double *orc_virialmol(orc *s) { return s->virialmol; }
int orc_np(orc *s) { return s->np; }
int orc_halo_np(orc *s) { return s->halo_np; }
int orc_iter(orc *s) { return s->iter; }
void orc_set_iter(orc *s, int iter) { s->iter = iter; }
void orc_set_integration_algorithm(orc *s, int ia) { s->integration_algorithm = ia; }
double orc_rmax(orc *s) { return s->rmax; }
int orc_rebuild_count(orc *s) { return s->rebuild_count; }
void orc_geometry(orc *s, int ncells[3], double cellside[3], double *rneighbr2, double *rcutoff2,
                  double *potshift)
{
    for (int k = 0; k < 3; k++) { ncells[k] = s->ncells[k]; cellside[k] = s->cellsidelength[k]; }
    *rneighbr2 = s->rneighbr2; *rcutoff2 = s->rcutoff2; *potshift = s->potshift;
}
void orc_macro(orc *s, double out[9])
{
    out[0] = s->vsum; out[1] = s->mv2sum; out[2] = s->temperature; out[3] = s->kinenergy;
    out[4] = s->potenergy; out[5] = s->totenergy; out[6] = s->pressure; out[7] = s->virial;
    out[8] = s->potenergysum;
}

/* ------------------------------------------------------------------------ */
/* linked lists (linklist.f90)                                               */
/* ------------------------------------------------------------------------ */

static inline int cidx(const orc *s, int i, int j, int k) /* 1-based cell indices */
{
    return (i - 1) + (s->ncells[0] + 2) * ((j - 1) + (s->ncells[1] + 2) * (k - 1));
}

/* linklist_deallocateall for the cell and neighbour lists
 * (linklist.f90:2872-2964). */
void orc_linklist_deallocateall(orc *s)
{
    if (s->potential_flag == 1) { /* linklist.f90:2889-2892 */
        memset(s->bond, 0, sizeof(int) * (size_t)s->max_funcy * (size_t)s->np);
        memset(s->bondcount, 0, sizeof(int) * (size_t)s->np);
    }
    memset(s->cellnp, 0, sizeof(int) * (size_t)s->ncell_tot);
    memset(s->cellhead, 0, sizeof(int) * (size_t)s->ncell_tot);
    s->cn_count = 0;
    memset(s->Nlist, 0, sizeof(int) * (size_t)s->np);
    memset(s->nhead, 0, sizeof(int) * (size_t)s->np);
    s->nn_count = 0;
}

/* linklist_checkpush (linklist.f90:1596-1632): head insert. */
static int checkpush(orc *s, int c, int molno)
{
    if (s->cn_count >= s->cn_cap) return ORC_ERR_ALLOC;
    int node = ++s->cn_count; /* 1-based node id, 0 = null */
    s->cn_molno[node - 1] = molno;
    s->cn_next[node - 1] = s->cellnp[c] > 0 ? s->cellhead[c] : 0;
    s->cellhead[c] = node;
    s->cellnp[c] += 1;
    return ORC_OK;
}

/* linklist_checkpushneighbr (linklist.f90:1636-1670): head insert into the
 * list of molnoi. */
static int checkpushneighbr(orc *s, int molnoi, int molnoj)
{
    if (s->nn_count >= s->nn_cap) {
        long ncap = s->nn_cap * 2;
        int *m = (int *)realloc(s->nn_molno, sizeof(int) * (size_t)ncap);
        if (!m) return ORC_ERR_ALLOC;
        s->nn_molno = m;
        int *x = (int *)realloc(s->nn_next, sizeof(int) * (size_t)ncap);
        if (!x) return ORC_ERR_ALLOC;
        s->nn_next = x;
        s->nn_cap = ncap;
    }
    long node = ++s->nn_count;
    s->nn_molno[node - 1] = molnoj;
    s->nn_next[node - 1] = s->Nlist[molnoi - 1] > 0 ? s->nhead[molnoi - 1] : 0;
    s->nhead[molnoi - 1] = (int)node;
    s->Nlist[molnoi - 1] += 1;
    return ORC_OK;
}

static inline int node_molno(const orc *s, int node) { return s->cn_molno[node - 1]; }
static inline int node_next(const orc *s, int node) { return s->cn_next[node - 1]; }

/* assign_to_cell (linklist.f90:2645-2679).  A molecule whose cell falls
 * outside 1..ncells+2 makes the reference abort ("escaped mol"). */
int orc_assign_to_cell(orc *s)
{
    for (int n = 1; n <= s->np; n++) {
        const double *rn = &s->r[3 * (size_t)(n - 1)];
        int ic = (int)ceil((rn[0] + s->halfdomain[0]) / s->cellsidelength[0]) + 1;
        int jc = (int)ceil((rn[1] + s->halfdomain[1]) / s->cellsidelength[1]) + 1;
        int kc = (int)ceil((rn[2] + s->halfdomain[2]) / s->cellsidelength[2]) + 1;
        if (ic < 1 || jc < 1 || kc < 1 || ic > s->ncells[0] + 2 || jc > s->ncells[1] + 2 ||
            kc > s->ncells[2] + 2)
            return ORC_ERR_ESCAPE;
        int rc = checkpush(s, cidx(s, ic, jc, kc), n);
        if (rc) return rc;
    }
    return ORC_OK;
}

/* assign_to_halocell (linklist.f90:2681-2706).  No escape check in the
 * reference; an image that bins outside the grid is reported here instead of
 * writing out of bounds. */
static int assign_to_halocell(orc *s, int start, int finish)
{
    for (int n = start; n <= finish; n++) {
        const double *rn = &s->r[3 * (size_t)(n - 1)];
        int ic = (int)ceil((rn[0] + s->halfdomain[0]) / s->cellsidelength[0]) + 1;
        int jc = (int)ceil((rn[1] + s->halfdomain[1]) / s->cellsidelength[1]) + 1;
        int kc = (int)ceil((rn[2] + s->halfdomain[2]) / s->cellsidelength[2]) + 1;
        if (ic < 1 || jc < 1 || kc < 1 || ic > s->ncells[0] + 2 || jc > s->ncells[1] + 2 ||
            kc > s->ncells[2] + 2)
            return ORC_ERR_ESCAPE;
        int rc = checkpush(s, cidx(s, ic, jc, kc), n);
        if (rc) return rc;
    }
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* halo images, single-rank periodic form (messenger.serial.f90:278-770)     */
/* ------------------------------------------------------------------------ */

static int add_image(orc *s, int molno, int sx, int sy, int sz)
{
    int m = s->np + s->halo_np + 1; /* 1-based index of the new image */
    if (m > s->cap) return ORC_ERR_ALLOC;
    double *dst = &s->r[3 * (size_t)(m - 1)];
    const double *src = &s->r[3 * (size_t)(molno - 1)];
    dst[0] = src[0]; dst[1] = src[1]; dst[2] = src[2];
    /* r(k,np+m) = r(k,np+m) +/- domain(k): one FP64 add per shifted axis */
    if (sx) dst[0] = dst[0] + (double)sx * s->domain[0];
    if (sy) dst[1] = dst[1] + (double)sy * s->domain[1];
    if (sz) dst[2] = dst[2] + (double)sz * s->domain[2];
    double *vd = &s->v[3 * (size_t)(m - 1)];
    const double *vs = &s->v[3 * (size_t)(molno - 1)];
    vd[0] = vs[0]; vd[1] = vs[1]; vd[2] = vs[2];
    s->glob_no[m - 1] = s->glob_no[molno - 1];
    s->halo_src[m - 1] = molno;
    s->halo_shift[3 * (size_t)(m - 1) + 0] = (signed char)sx;
    s->halo_shift[3 * (size_t)(m - 1) + 1] = (signed char)sy;
    s->halo_shift[3 * (size_t)(m - 1) + 2] = (signed char)sz;
    s->chainID[m - 1] = s->chainID[molno - 1];
    s->subchainID[m - 1] = s->subchainID[molno - 1];
    s->funcy[m - 1] = s->funcy[molno - 1];
    for (int b = 0; b < 4; b++) s->bflag[4 * (size_t)(m - 1) + b] = s->bflag[4 * (size_t)(molno - 1) + b];
    s->halo_np += 1;
    return ORC_OK;
}

static int image_cell(orc *s, int i, int j, int k, int sx, int sy, int sz)
{
    int c = cidx(s, i, j, k);
    int node = s->cellhead[c];
    for (int n = 0; n < s->cellnp[c]; n++) {
        int rc = add_image(s, node_molno(s, node), sx, sy, sz);
        if (rc) return rc;
        node = node_next(s, node);
    }
    return ORC_OK;
}

/* sign(1, x) in Fortran: +1 for x >= 0 */
static inline int fsign1(int x) { return x >= 0 ? 1 : -1; }

/* messenger_updateborders_quiescent (messenger.serial.f90:278-323) with
 * updatefacedown/up (372-584), updateedge (589-710), updatecorners (715-770). */
int orc_updateborders(orc *s, int rebuild)
{
    const int nx = s->ncells[0], ny = s->ncells[1], nz = s->ncells[2];
    int rc;
    s->halo_np = 0;
    /* faces down (+domain) then up (-domain), x, y, z */
    for (int ixyz = 0; ixyz < 3; ixyz++) {
        for (int dir = 0; dir < 2; dir++) {
            int sgn = dir == 0 ? +1 : -1;
            if (ixyz == 0) {
                int ic = dir == 0 ? 2 : nx + 1;
                for (int jc = 2; jc <= ny + 1; jc++)
                    for (int kc = 2; kc <= nz + 1; kc++)
                        if ((rc = image_cell(s, ic, jc, kc, sgn, 0, 0))) return rc;
            } else if (ixyz == 1) {
                int jc = dir == 0 ? 2 : ny + 1;
                for (int ic = 2; ic <= nx + 1; ic++)
                    for (int kc = 2; kc <= nz + 1; kc++)
                        if ((rc = image_cell(s, ic, jc, kc, 0, sgn, 0))) return rc;
            } else {
                int kc = dir == 0 ? 2 : nz + 1;
                for (int ic = 2; ic <= nx + 1; ic++)
                    for (int jc = 2; jc <= ny + 1; jc++)
                        if ((rc = image_cell(s, ic, jc, kc, 0, 0, sgn))) return rc;
            }
        }
    }
    /* edges: updateedge(1,2) -> along z, (2,3) -> along x, (1,3) -> along y */
    const int order[3] = {2, 0, 1};
    for (int e = 0; e < 3; e++) {
        int ixyz = order[e];
        if (ixyz == 0) { /* edge1 over y, edge2 over z */
            int e1[4] = {2, 2, ny + 1, ny + 1}, e2[4] = {2, nz + 1, 2, nz + 1};
            for (int q = 0; q < 4; q++)
                for (int ic = 2; ic <= nx + 1; ic++)
                    if ((rc = image_cell(s, ic, e1[q], e2[q], 0, fsign1(ny - e1[q]), fsign1(nz - e2[q]))))
                        return rc;
        } else if (ixyz == 1) { /* edge1 over x, edge2 over z */
            int e1[4] = {2, 2, nx + 1, nx + 1}, e2[4] = {2, nz + 1, 2, nz + 1};
            for (int q = 0; q < 4; q++)
                for (int jc = 2; jc <= ny + 1; jc++)
                    if ((rc = image_cell(s, e1[q], jc, e2[q], fsign1(nx - e1[q]), 0, fsign1(nz - e2[q]))))
                        return rc;
        } else { /* edge1 over x, edge2 over y */
            int e1[4] = {2, 2, nx + 1, nx + 1}, e2[4] = {2, ny + 1, 2, ny + 1};
            for (int q = 0; q < 4; q++)
                for (int kc = 2; kc <= nz + 1; kc++)
                    if ((rc = image_cell(s, e1[q], e2[q], kc, fsign1(nx - e1[q]), fsign1(ny - e2[q]), 0)))
                        return rc;
        }
    }
    /* corners */
    {
        int ci[8] = {2, 2, 2, 2, nx + 1, nx + 1, nx + 1, nx + 1};
        int cj[8] = {2, 2, ny + 1, ny + 1, 2, 2, ny + 1, ny + 1};
        int ck[8] = {2, nz + 1, 2, nz + 1, 2, nz + 1, 2, nz + 1};
        for (int q = 0; q < 8; q++)
            if ((rc = image_cell(s, ci[q], cj[q], ck[q], fsign1(nx - ci[q]), fsign1(ny - cj[q]),
                                 fsign1(nz - ck[q]))))
                return rc;
    }
    if (rebuild == 1) return assign_to_halocell(s, s->np + 1, s->np + s->halo_np);
    return ORC_OK;
}

/* Refresh image positions from their sources without re-walking the cells.
 * Equivalent to messenger_updateborders(0) because the cell lists (and hence
 * the image order) only change on rebuild. */
void orc_refresh_halo(orc *s)
{
    for (int m = s->np + 1; m <= s->np + s->halo_np; m++) {
        int src = s->halo_src[m - 1];
        for (int k = 0; k < 3; k++) {
            double x = s->r[3 * (size_t)(src - 1) + k];
            int sh = s->halo_shift[3 * (size_t)(m - 1) + k];
            if (sh) x = x + (double)sh * s->domain[k];
            s->r[3 * (size_t)(m - 1) + k] = x;
            s->v[3 * (size_t)(m - 1) + k] = s->v[3 * (size_t)(src - 1) + k];
        }
    }
}

/* ------------------------------------------------------------------------ */
/* polymer bond discovery (linklist.f90:2542-2584, modules.f90:597-610)      */
/* ------------------------------------------------------------------------ */

/* get_bondflag (modules.f90:602-610): subchain scID maps to word
 * ceiling(scID/31) and bit mod(scID,31)-1 (bit 30 when that is -1), with
 * intbits = bit_size(1)-1 = 31 (modules.f90:497). */
static int get_bondflag(const orc *s, int i, int subj)
{
    int ipos = subj - 1;
    int group = ipos / 31;
    int expo = ipos % 31;
    if (group < 0 || group > 3) return 0;
    return (s->bflag[4 * (size_t)(i - 1) + group] >> expo) & 1;
}

static int check_update_adjacentbeadinfo(orc *s, int molnoi, int molnoj)
{
    if (s->chainID[molnoi - 1] != s->chainID[molnoj - 1] || s->chainID[molnoi - 1] == 0) return ORC_OK;
    int bflag = get_bondflag(s, molnoi, s->subchainID[molnoj - 1]);
    if (!bflag) return ORC_OK;
    /* bond(bondcount+1, i) = j on both partners (linklist.f90:2556-2565); only
     * the real molecules' rows are ever read by the force loop */
    if (molnoi <= s->np) {
        int bc = s->bondcount[molnoi - 1];
        if (bc >= s->max_funcy) return ORC_ERR_BOND;
        s->bond[(size_t)(molnoi - 1) * s->max_funcy + bc] = molnoj;
        s->bondcount[molnoi - 1] = bc + 1;
    }
    if (molnoj <= s->np) {
        int bc = s->bondcount[molnoj - 1];
        if (bc >= s->max_funcy) return ORC_ERR_BOND;
        s->bond[(size_t)(molnoj - 1) * s->max_funcy + bc] = molnoi;
        s->bondcount[molnoj - 1] = bc + 1;
    }
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* neighbour lists                                                           */
/* ------------------------------------------------------------------------ */

static inline double rij2_of(const orc *s, int mi, int mj, double rij[3])
{
    const double *ri = &s->r[3 * (size_t)(mi - 1)];
    const double *rj = &s->r[3 * (size_t)(mj - 1)];
    rij[0] = ri[0] - rj[0];
    rij[1] = ri[1] - rj[1];
    rij[2] = ri[2] - rj[2];
    double d = 0.0;
    d = d + rij[0] * rij[0];
    d = d + rij[1] * rij[1];
    d = d + rij[2] * rij[2];
    return d;
}

/* calculate_cell_interactions_opt (linklist.f90:1118-1180): pairs between a
 * halo cell range and its shifted neighbour, stored on molnoj's list. */
static int cell_interactions_opt(orc *s, int is, int ie, int ish, int js, int je, int jsh, int ks,
                                 int ke, int ksh)
{
    double rij[3];
    int rc;
    for (int kc = ks; kc <= ke; kc++)
        for (int jc = js; jc <= je; jc++)
            for (int ic = is; ic <= ie; ic++) {
                int c = cidx(s, ic, jc, kc);
                int c2 = cidx(s, ic + ish, jc + jsh, kc + ksh);
                int oldi = s->cellhead[c];
                for (int i = 0; i < s->cellnp[c]; i++) {
                    int molnoi = node_molno(s, oldi);
                    int oldj = s->cellhead[c2];
                    for (int j = 0; j < s->cellnp[c2]; j++) {
                        int molnoj = node_molno(s, oldj);
                        oldj = node_next(s, oldj);
                        double r2 = rij2_of(s, molnoi, molnoj, rij);
                        if (s->potential_flag == 1)
                            if ((rc = check_update_adjacentbeadinfo(s, molnoi, molnoj))) return rc;
                        if (r2 < s->rneighbr2)
                            if ((rc = checkpushneighbr(s, molnoj, molnoi))) return rc;
                    }
                    oldi = node_next(s, oldi);
                }
            }
    return ORC_OK;
}

static const int ISH[13] = {1, 1, 0, -1, 0, 1, 1, 0, -1, -1, -1, 0, 1};
static const int JSH[13] = {0, 1, 1, 1, 0, 0, 1, 1, 1, 0, -1, -1, -1};
static const int KSH[13] = {0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 1, 1, 1};

/* assign_to_neighbourlist_halfint_opt (linklist.f90:660-804). */
int orc_neighbourlist_halfint_opt(orc *s)
{
    const int nx = s->ncells[0], ny = s->ncells[1], nz = s->ncells[2];
    double rij[3];
    int rc;
    memset(s->Nlist, 0, sizeof(int) * (size_t)s->np);
    memset(s->nhead, 0, sizeof(int) * (size_t)s->np);
    s->nn_count = 0;
    for (int ic = 2; ic <= nx + 1; ic++)
        for (int jc = 2; jc <= ny + 1; jc++)
            for (int kc = 2; kc <= nz + 1; kc++) {
                int c = cidx(s, ic, jc, kc);
                int cellnp = s->cellnp[c];
                int oldi = s->cellhead[c];
                for (int i = 1; i <= cellnp; i++) { /* own cell, j after i */
                    int molnoi = node_molno(s, oldi);
                    int oldj = node_next(s, oldi);
                    for (int j = i + 1; j <= cellnp; j++) {
                        int molnoj = node_molno(s, oldj);
                        oldj = node_next(s, oldj);
                        if (molnoi == molnoj) continue;
                        double r2 = rij2_of(s, molnoi, molnoj, rij);
                        if (s->potential_flag == 1)
                            if ((rc = check_update_adjacentbeadinfo(s, molnoi, molnoj))) return rc;
                        if (r2 < s->rneighbr2)
                            if ((rc = checkpushneighbr(s, molnoi, molnoj))) return rc;
                    }
                    oldi = node_next(s, oldi);
                }
                int oldihead = s->cellhead[c];
                for (int k = 0; k < 13; k++) {
                    int c2 = cidx(s, ic + ISH[k], jc + JSH[k], kc + KSH[k]);
                    int oldi2 = oldihead;
                    for (int i = 0; i < cellnp; i++) {
                        int molnoi = node_molno(s, oldi2);
                        int oldj = s->cellhead[c2];
                        for (int j = 0; j < s->cellnp[c2]; j++) {
                            int molnoj = node_molno(s, oldj);
                            oldj = node_next(s, oldj);
                            double r2 = rij2_of(s, molnoi, molnoj, rij);
                            if (s->potential_flag == 1)
                                if ((rc = check_update_adjacentbeadinfo(s, molnoi, molnoj))) return rc;
                            if (r2 < s->rneighbr2)
                                if ((rc = checkpushneighbr(s, molnoi, molnoj))) return rc;
                        }
                        oldi2 = node_next(s, oldi2);
                    }
                }
            }
    /* all_cell_interactions (linklist.f90:778-802): 27 sweeps from halo cells */
    {
        int x = nx, x1 = nx + 1, x2 = nx + 2, y = ny, y1 = ny + 1, y2 = ny + 2, z = nz, z1 = nz + 1;
        const int imin[27] = {2, 1, 3, 2, 2, 1, 3, 3, 1, 1, 1, 1, 1, 1, x2, x2, x2, x2, 2, 2, 3, 2, 2, 3, 2, 3, 2};
        const int imax[27] = {x1, x, x2, x1, x1, x, x2, x2, x, 1, 1, 1, 1, 1, x2, x2, x2, x2, x1, x, x1, x1, x, x1, x1, x1, x};
        const int jmin[27] = {2, 2, 2, 1, 3, 1, 1, 3, 3, 2, 2, 1, 1, 3, 1, 2, 1, 3, 1, 1, 1, 1, 1, 1, y2, y2, y2};
        const int jmax[27] = {y1, y1, y1, y, y2, y, y, y2, y2, y1, y1, y, y, y2, y, y1, y, y2, 1, 1, 1, 1, 1, 1, y2, y2, y2};
        const int kmin[27] = {1, 1, 1, 1, 1, 1, 1, 1, 1, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2};
        const int kmax[27] = {1, 1, 1, 1, 1, 1, 1, 1, 1, z1, z, z1, z, z, z1, z, z, z, z1, z1, z1, z, z, z, z, z, z};
        const int shift[27] = {5, 6, 10, 8, 12, 7, 9, 11, 13, 1, 6, 2, 7, 13, 4, 10, 9, 11, 3, 2, 4, 8, 7, 9, 12, 11, 13};
        for (int q = 0; q < 27; q++) {
            int sh = shift[q] - 1;
            if ((rc = cell_interactions_opt(s, imin[q], imax[q], ISH[sh], jmin[q], jmax[q], JSH[sh], kmin[q],
                                            kmax[q], KSH[sh])))
                return rc;
        }
    }
    return ORC_OK;
}

/* assign_to_neighbourlist_allint (linklist.f90:181-263). */
int orc_neighbourlist_allint(orc *s)
{
    double rij[3];
    int rc;
    memset(s->Nlist, 0, sizeof(int) * (size_t)s->np);
    memset(s->nhead, 0, sizeof(int) * (size_t)s->np);
    s->nn_count = 0;
    for (int ic = 2; ic <= s->ncells[0] + 1; ic++)
        for (int jc = 2; jc <= s->ncells[1] + 1; jc++)
            for (int kc = 2; kc <= s->ncells[2] + 1; kc++) {
                int c = cidx(s, ic, jc, kc);
                int oldi = s->cellhead[c];
                for (int i = 0; i < s->cellnp[c]; i++) {
                    int molnoi = node_molno(s, oldi);
                    for (int di = -1; di <= 1; di++)
                        for (int dj = -1; dj <= 1; dj++)
                            for (int dk = -1; dk <= 1; dk++) {
                                int c2 = cidx(s, ic + di, jc + dj, kc + dk);
                                int oldj = s->cellhead[c2];
                                for (int j = 0; j < s->cellnp[c2]; j++) {
                                    int molnoj = node_molno(s, oldj);
                                    oldj = node_next(s, oldj);
                                    if (molnoi == molnoj) continue;
                                    double r2 = rij2_of(s, molnoi, molnoj, rij);
                                    if (r2 < s->rneighbr2)
                                        if ((rc = checkpushneighbr(s, molnoi, molnoj))) return rc;
                                }
                            }
                    oldi = node_next(s, oldi);
                }
            }
    return ORC_OK;
}

/* assign_to_neighbourlist (linklist.f90:2710-2741). */
int orc_assign_to_neighbourlist(orc *s)
{
    if (s->force_list == 2) return orc_neighbourlist_allint(s);
    if (s->force_list == 3) return orc_neighbourlist_halfint_opt(s);
    return ORC_OK;
}

/* Exports the list as (owner, partner-source, shift-code) with 1-based
 * glob_no identities; shift code = (sx+1) + 3(sy+1) + 9(sz+1), 13 = none. */
long orc_pair_list(orc *s, int *owner, int *partner, int *code, long cap)
{
    long n = 0;
    for (int i = 1; i <= s->np; i++) {
        int node = s->nhead[i - 1];
        for (int q = 0; q < s->Nlist[i - 1]; q++) {
            int j = s->nn_molno[node - 1];
            node = s->nn_next[node - 1];
            if (n < cap) {
                owner[n] = s->glob_no[i - 1];
                if (j <= s->np) {
                    partner[n] = s->glob_no[j - 1];
                    code[n] = 13;
                } else {
                    const signed char *sh = &s->halo_shift[3 * (size_t)(j - 1)];
                    partner[n] = s->glob_no[s->halo_src[j - 1] - 1];
                    code[n] = (sh[0] + 1) + 3 * (sh[1] + 1) + 9 * (sh[2] + 1);
                }
            }
            n++;
        }
    }
    return n;
}

long orc_list_length(orc *s) { return s->nn_count; }

/* ------------------------------------------------------------------------ */
/* forces (simulation_compute_forces.f90)                                    */
/* ------------------------------------------------------------------------ */

static void zero_forces(orc *s)
{
    size_t tot = (size_t)(s->np + s->halo_np);
    memset(s->a, 0, sizeof(double) * 3 * tot);
    memset(s->potenergymol, 0, sizeof(double) * tot);
    memset(s->potenergymol_POLY, 0, sizeof(double) * tot);
    memset(s->virialmol, 0, sizeof(double) * tot);
    if (s->pressure_outflag) memset(s->rfmol, 0, sizeof(double) * 9 * tot);
    s->virial = 0.0;
}

/* pressure_tensor_forces (simulation_record.f90:6239-6256). */
static inline void ptf(orc *s, int molno, const double rij[3], double acc)
{
    double *rf = &s->rfmol[9 * (size_t)(molno - 1)];
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) rf[3 * a + b] = rf[3 * a + b] + acc * rij[a] * rij[b];
}

/* simulation_compute_forces_LJ_neigbr_halfint (:628-726). */
static void forces_halfint(orc *s)
{
    const int rec = (s->iter % s->tplot) == 0;
    const int tev = (s->iter % s->teval) == 0;
    double rij[3];
    for (int i = 1; i <= s->np; i++) {
        int node = s->nhead[i - 1];
        for (int q = 0; q < s->Nlist[i - 1]; q++) {
            int j = s->nn_molno[node - 1];
            node = s->nn_next[node - 1];
            double r2 = rij2_of(s, i, j, rij);
            if (r2 < s->rcutoff2) {
                double inv = 1.0 / r2;
                double acc = pair_accijmag(s, inv, i, j);
                double mi = mass_of(s, i), mj = mass_of(s, j);
                double *ai = &s->a[3 * (size_t)(i - 1)], *aj = &s->a[3 * (size_t)(j - 1)];
                ai[0] = ai[0] + acc * rij[0] / mi;
                ai[1] = ai[1] + acc * rij[1] / mi;
                ai[2] = ai[2] + acc * rij[2] / mi;
                aj[0] = aj[0] - acc * rij[0] / mj;
                aj[1] = aj[1] - acc * rij[1] / mj;
                aj[2] = aj[2] - acc * rij[2] / mj;
                if (rec) {
                    double e = pair_energy(s, inv, i, j);
                    s->potenergymol[i - 1] += e;
                    s->potenergymol[j - 1] += e;
                    s->virialmol[i - 1] += acc * r2;
                    s->virialmol[j - 1] += acc * r2;
                    if (s->pressure_outflag == 1) { /* :698-701 */
                        ptf(s, i, rij, acc);
                        if (j <= s->np) ptf(s, j, rij, acc);
                    }
                } else if (tev) {
                    s->virialmol[i - 1] += acc * r2;
                    s->virialmol[j - 1] += acc * r2;
                }
            }
        }
    }
}

/* simulation_compute_forces_Soddemann_neigbr_halfint (:793-888): half list;
 * WCA (get_accijmag: LJ_accijmag, or Mie_accijmag of the pair's types with
 * Mie_potential 1; the energy is the LJ-WCA expression either way) below
 * wca_cut2 and the reference's cosine-well
 * expression out to sod_cut2, the well depth by how many of the pair are
 * chain beads (chainID != 0; an image has its source's).  The minimum-image
 * line (:821) leaves rij as it is for every listed pair (|rij| < L/2, as
 * there are at least 3 cells of rcutoff + delta per axis), so it is not
 * repeated.  Accelerations are not divided by a mass (:852-860); no
 * pressure-tensor term is recorded (the routine calls none). */
static void forces_soddemann(orc *s)
{
    const int rec = (s->iter % s->tplot) == 0;
    const int tev = (s->iter % s->teval) == 0;
    const double A = sod_a(), B = sod_b(), W2 = wca_cut2();
    double rij[3];
    for (int i = 1; i <= s->np; i++) {
        int node = s->nhead[i - 1];
        for (int q = 0; q < s->Nlist[i - 1]; q++) {
            int j = s->nn_molno[node - 1];
            node = s->nn_next[node - 1];
            double r2 = rij2_of(s, i, j, rij);
            if (!(r2 < SOD_CUT2)) continue;
            const int ptot = (s->chainID[i - 1] != 0) + (s->chainID[j - 1] != 0);
            const double eps = s->sod_eps[ptot];
            const double inv = 1.0 / r2;
            double acc;
            if (r2 < W2) acc = pair_accijmag(s, inv, i, j); /* get_accijmag (:839) */
            else acc = (eps * A * (inv * inv)) * sin(inv * A + B);
            double *ai = &s->a[3 * (size_t)(i - 1)], *aj = &s->a[3 * (size_t)(j - 1)];
            for (int k = 0; k < 3; k++) {
                ai[k] = ai[k] + acc * rij[k];
                aj[k] = aj[k] - acc * rij[k];
            }
            if (rec) {
                double e = r2 < W2 ? 4.0 * (p6(inv) - p3(inv) + 0.25) - eps : 0.5 * eps * (cos(A * r2 + B) - 1.0);
                s->potenergymol[i - 1] += e;
                s->potenergymol[j - 1] += e;
                s->virialmol[i - 1] += acc * r2;
                s->virialmol[j - 1] += acc * r2;
            } else if (tev) {
                s->virialmol[i - 1] += acc * r2;
                s->virialmol[j - 1] += acc * r2;
            }
        }
    }
}

/* simulation_compute_forces_LJ_neigbr (:551-623): full list, i side only. */
static void forces_full(orc *s)
{
    const int rec = (s->iter % s->tplot) == 0;
    const int tev = (s->iter % s->teval) == 0;
    double rij[3];
    for (int i = 1; i <= s->np; i++) {
        int node = s->nhead[i - 1];
        for (int q = 0; q < s->Nlist[i - 1]; q++) {
            int j = s->nn_molno[node - 1];
            node = s->nn_next[node - 1];
            double r2 = rij2_of(s, i, j, rij);
            if (r2 < s->rcutoff2) {
                double inv = 1.0 / r2;
                double acc = pair_accijmag(s, inv, i, j);
                double mi = mass_of(s, i);
                double *ai = &s->a[3 * (size_t)(i - 1)];
                ai[0] = ai[0] + acc * rij[0] / mi;
                ai[1] = ai[1] + acc * rij[1] / mi;
                ai[2] = ai[2] + acc * rij[2] / mi;
                if (rec) {
                    s->potenergymol[i - 1] += pair_energy(s, inv, i, j);
                    s->virialmol[i - 1] += acc * r2;
                    if (s->pressure_outflag == 1) ptf(s, i, rij, acc); /* :603 */
                } else if (tev) {
                    s->virialmol[i - 1] += acc * r2;
                }
            }
        }
    }
}

/* simulation_compute_forces_LJ_AP (:280-341): all pairs, per-axis minimum
 * image.  The routine records no pressure-tensor term. */
static void forces_AP(orc *s)
{
    const int rec = (s->iter % s->tplot) == 0;
    const int tev = (s->iter % s->teval) == 0;
    double rij[3];
    for (int i = 1; i <= s->np; i++) {
        const double *ri = &s->r[3 * (size_t)(i - 1)];
        for (int j = i + 1; j <= s->np; j++) {
            const double *rj = &s->r[3 * (size_t)(j - 1)];
            double r2 = 0.0;
            for (int k = 0; k < 3; k++) {
                rij[k] = ri[k] - rj[k];
                if (fabs(rij[k]) > s->halfdomain[k]) rij[k] = rij[k] - copysign(s->domain[k], rij[k]);
                r2 = r2 + rij[k] * rij[k];
            }
            if (r2 < s->rcutoff2) {
                double inv = 1.0 / r2;
                double acc = pair_accijmag(s, inv, i, j);
                double mi = mass_of(s, i), mj = mass_of(s, j);
                double *ai = &s->a[3 * (size_t)(i - 1)], *aj = &s->a[3 * (size_t)(j - 1)];
                for (int k = 0; k < 3; k++) {
                    ai[k] = ai[k] + acc * rij[k] / mi;
                    aj[k] = aj[k] - acc * rij[k] / mj;
                }
                if (rec) {
                    double e = pair_energy(s, inv, i, j);
                    s->potenergymol[i - 1] += e;
                    s->potenergymol[j - 1] += e;
                    s->virialmol[i - 1] += acc * r2;
                    s->virialmol[j - 1] += acc * r2;
                } else if (tev) {
                    s->virialmol[i - 1] += acc * r2;
                    s->virialmol[j - 1] += acc * r2;
                }
            }
        }
    }
}

/* simulation_compute_forces_poly (:731-789): bonded FENE, i side only. */
static int forces_poly(orc *s)
{
    const int rec = (s->iter % s->tplot) == 0;
    const int tev = (s->iter % s->teval) == 0;
    double rij[3];
    for (int i = 1; i <= s->np; i++) {
        for (int b = 0; b < s->funcy[i - 1] && b < s->max_funcy; b++) {
            int j = s->bond[(size_t)(i - 1) * s->max_funcy + b];
            if (j == 0) continue;
            double r2 = rij2_of(s, i, j, rij);
            double acc;
            if (s->mie) {
                acc = harmonic_accijmag(s, r2, i, j); /* get_poly_accijmag => harmonic (:1215) */
            } else {
                if (r2 >= s->R_0 * s->R_0) return ORC_ERR_BOND; /* polymer_bond_error */
                acc = fene_accijmag(r2, s->k_c, s->R_0);
            }
            double mi = mass_of(s, i);
            double *ai = &s->a[3 * (size_t)(i - 1)];
            ai[0] = ai[0] + acc * rij[0] / mi;
            ai[1] = ai[1] + acc * rij[1] / mi;
            ai[2] = ai[2] + acc * rij[2] / mi;
            if (rec) {
                if (s->pressure_outflag == 1) ptf(s, i, rij, acc); /* :768-770 */
                s->potenergymol_POLY[i - 1] += s->mie ? harmonic_energy(s, r2, i, j) : fene_energy(r2, s->k_c, s->R_0);
                s->virialmol[i - 1] += acc * r2;
            } else if (tev) {
                s->virialmol[i - 1] += acc * r2;
            }
        }
    }
    return ORC_OK;
}

/* simulation_compute_forces_angular (simulation_compute_forces.f90:981-1048)
 * with angular_harmonic_force (setup_set_parameters.f90:441-489), for every
 * real middle bead j (funcy 2): i = bond(1,j), k = bond(2,j) in the order the
 * list build discovered the bonds (a cross-boundary partner is its halo
 * image), rij = r_i - r_j, rjk = r_j - r_k, theta = acos(rij.rjk/(|rij||rjk|)),
 *   aForce(1) = -(k (theta - theta_0) / (|rij| sin theta)) (rjk/|rjk| - rij/|rij| cos theta)
 *   aForce(3) = -(k (theta - theta_0) / (|rjk| sin theta)) (rij/|rij| - rjk/|rjk| cos theta)
 *   aForce(2) = -aForce(1) - aForce(3), zero when theta < 1e-5,
 * and a(i) -= aForce(1)/m_i, a(j) -= aForce(2)/m_j, a(k) -= aForce(3)/m_k
 * (the rows of halo images are not returned).  No energy is recorded.
 * Where the reference has no defined result this returns ORC_ERR_BOND: a
 * middle bead without both bonds (its fallbacks read bond(3:4) or a stale
 * index), a triple whose k_ijk < 1e-5 (the function returns its result
 * unset), and a middle bead that has a halo image (the reference also loops
 * over halo beads, whose bond rows hold only the partners found from interior
 * cells). */
static int forces_angular(orc *s)
{
    const int nt = s->ang_nt;
    for (int n = s->np + 1; n <= s->np + s->halo_np; n++)
        if (s->funcy[s->halo_src[n - 1] - 1] == 2) return ORC_ERR_BOND;
    for (int j = 1; j <= s->np; j++) {
        if (s->funcy[j - 1] != 2) continue;
        const int i = s->bond[(size_t)(j - 1) * s->max_funcy + 0];
        const int k = s->bond[(size_t)(j - 1) * s->max_funcy + 1];
        if (i == 0 || k == 0) return ORC_ERR_BOND;
        const int q = (type_of(s, i) - 1) + nt * ((type_of(s, j) - 1) + nt * (type_of(s, k) - 1));
        const double kk = s->ang_k[q], t0 = s->ang_t0[q];
        if (kk < 1e-5) return ORC_ERR_BOND;
        const double *ri = &s->r[3 * (size_t)(i - 1)], *rj = &s->r[3 * (size_t)(j - 1)],
                     *rk = &s->r[3 * (size_t)(k - 1)];
        double rij[3], rjk[3];
        for (int c = 0; c < 3; c++) { rij[c] = ri[c] - rj[c]; rjk[c] = rj[c] - rk[c]; }
        const double mag_ij = sqrt(rij[0] * rij[0] + rij[1] * rij[1] + rij[2] * rij[2]);
        const double mag_jk = sqrt(rjk[0] * rjk[0] + rjk[1] * rjk[1] + rjk[2] * rjk[2]);
        const double th = acos((rij[0] * rjk[0] + rij[1] * rjk[1] + rij[2] * rjk[2]) / (mag_ij * mag_jk));
        double f1[3] = {0.0, 0.0, 0.0}, f3[3] = {0.0, 0.0, 0.0}, f2[3];
        if (!(th < 1e-5)) {
            const double ct = cos(th), st = sin(th);
            const double c1 = kk * (th - t0) / (mag_ij * st), c3 = kk * (th - t0) / (mag_jk * st);
            for (int c = 0; c < 3; c++) {
                f1[c] = -c1 * (rjk[c] / mag_jk - rij[c] / mag_ij * ct);
                f3[c] = -c3 * (rij[c] / mag_ij - rjk[c] / mag_jk * ct);
            }
        }
        for (int c = 0; c < 3; c++) f2[c] = -f1[c] - f3[c];
        const double mi = mass_of(s, i), mj = mass_of(s, j), mk = mass_of(s, k);
        double *ai = &s->a[3 * (size_t)(i - 1)], *aj = &s->a[3 * (size_t)(j - 1)], *ak = &s->a[3 * (size_t)(k - 1)];
        for (int c = 0; c < 3; c++) {
            ai[c] = ai[c] - f1[c] / mi;
            aj[c] = aj[c] - f2[c] / mj;
            ak[c] = ak[c] - f3[c] / mk;
        }
    }
    return ORC_OK;
}

/* angular_potential on (simulation_compute_forces.f90:257-259: force_list 3,
 * potential_flag 1, solvent_flag 0); the types are the Mie moltypes. */
int orc_set_angular(orc *s, int ntypes, const double *k, const double *theta0)
{
    if (!s->mie || ntypes < 1 || ntypes > MIET) return ORC_ERR_PARAM;
    if (s->force_list != 3 || s->potential_flag != 1 || s->solvent_flag != 0) return ORC_ERR_PARAM;
    size_t n3 = (size_t)ntypes * ntypes * ntypes;
    free(s->ang_k); free(s->ang_t0);
    s->ang_k = (double *)xcalloc(n3, sizeof(double));
    s->ang_t0 = (double *)xcalloc(n3, sizeof(double));
    memcpy(s->ang_k, k, n3 * sizeof(double));
    memcpy(s->ang_t0, theta0, n3 * sizeof(double));
    s->ang_nt = ntypes;
    s->angular = 1;
    return ORC_OK;
}

/* simulation_compute_forces dispatcher (:182-275). */
int orc_compute_forces(orc *s)
{
    zero_forces(s);
    switch (s->force_list) {
    case 0: forces_AP(s); break;
    case 2: forces_full(s); break;
    case 3:
        if (s->potential_flag == 1 && s->solvent_flag == 1) forces_soddemann(s); /* :264-267 */
        else forces_halfint(s);
        break;
    default: return ORC_ERR_PARAM;
    }
    if (s->potential_flag == 1) {
        int rc = forces_poly(s);
        if (rc) return rc;
        for (int n = 0; n < s->np + s->halo_np; n++) s->potenergymol[n] += s->potenergymol_POLY[n];
        if (s->angular && s->force_list == 3 && s->solvent_flag == 0 && (rc = forces_angular(s))) return rc;
    }
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* integration (simulation_move_particles_vv.f90, NVE)                       */
/* ------------------------------------------------------------------------ */

void orc_move_vv(orc *s, int pass_num)
{
    const double dt = s->delta_t;
    const double c = 0.5 * (dt * dt);
    const double h = 0.5 * dt;
    if (pass_num == 1) { /* :64-69 */
        for (int n = 0; n < s->np; n++)
            for (int k = 0; k < 3; k++) {
                size_t q = 3 * (size_t)n + k;
                s->r[q] = s->r[q] + dt * s->v[q] + c * s->a[q];
                s->v[q] = s->v[q] + h * s->a[q];
            }
    } else { /* :132-135, simtime :191 */
        for (int n = 0; n < s->np; n++)
            for (int k = 0; k < 3; k++) {
                size_t q = 3 * (size_t)n + k;
                s->v[q] = s->v[q] + h * s->a[q];
            }
        s->simtime = s->simtime + dt;
    }
}

/* simulation_move_particles_lfv NVE (simulation_move_particles_lfv.f90:81-92). */
void orc_move_lfv(orc *s)
{
    const double dt = s->delta_t;
    for (int n = 0; n < s->np; n++)
        for (int k = 0; k < 3; k++) {
            size_t q = 3 * (size_t)n + k;
            s->v[q] = s->v[q] + dt * s->a[q];
            s->r[q] = s->r[q] + dt * s->v[q];
        }
    s->simtime = s->simtime + dt;
}

/* ------------------------------------------------------------------------ */
/* rebuild criterion (simulation_checkrebuild.f90:17-148)                    */
/* ------------------------------------------------------------------------ */

int orc_checkrebuild(orc *s)
{
    int rebuild = 0;
    if (((s->iter + 1) % s->tplot) == 0) rebuild = 1; /* :34 */
    double dmin = s->delta_rneighbr[0];
    if (s->delta_rneighbr[1] < dmin) dmin = s->delta_rneighbr[1];
    if (s->delta_rneighbr[2] < dmin) dmin = s->delta_rneighbr[2];
    if (s->rebuild_criteria == 0) { /* :84-99 */
        double vmax = 0.0;
        for (int n = 0; n < s->np; n++) {
            const double *vn = &s->v[3 * (size_t)n];
            double m = 0.0;
            m = m + vn[0] * vn[0];
            m = m + vn[1] * vn[1];
            m = m + vn[2] * vn[2];
            if (n == 0 || m > vmax) vmax = m;
        }
        vmax = sqrt(vmax);
        s->rmax = s->rmax + vmax * s->delta_t;
        if (s->rmax > 0.5 * dmin) rebuild = 1;
    } else if (s->rebuild_criteria == 1) { /* :101-103 */
        if ((s->iter % s->fixed_rebuild) == 0) rebuild = 1;
    } else { /* :105-121 */
        if (!s->rdisp) s->rdisp = (double *)xcalloc(3 * (size_t)s->np, sizeof(double));
        for (int n = 0; n < s->np; n++) {
            int hit = 0;
            for (int k = 0; k < 3; k++) {
                size_t q = 3 * (size_t)n + k;
                s->rdisp[q] = s->rdisp[q] + s->v[q] * s->delta_t;
                if (fabs(s->rdisp[q]) > 0.5 * dmin) hit = 1;
            }
            if (hit) { rebuild = 1; break; }
        }
    }
    if (rebuild) {
        s->rmax = 0.0;
        if (s->rebuild_criteria == 2 && s->rdisp) memset(s->rdisp, 0, sizeof(double) * 3 * (size_t)s->np);
        s->rebuild_count++;
    }
    return rebuild;
}

/* ------------------------------------------------------------------------ */
/* periodic wrap on rebuild (messenger.serial.f90:961-1028, in place)        */
/* ------------------------------------------------------------------------ */

static int is_teth(int t) { return t == 3 || t == 5 || t == 6 || t == 7; }

void orc_sendmols(orc *s)
{
    for (int n = 0; n < s->np; n++)
        for (int k = 0; k < 3; k++) {
            size_t q = 3 * (size_t)n + k;
            /* rtether moves with its molecule (messenger.serial.f90:971-1019) */
            int teth = s->ensemble == 6 && is_teth(s->tag[n]);
            if (s->r[q] >= s->halfdomain[k]) {
                s->r[q] = s->r[q] - s->domain[k];
                if (teth) s->rtether[q] = s->rtether[q] - s->domain[k];
            }
            if (s->r[q] < -s->halfdomain[k]) {
                s->r[q] = s->r[q] + s->domain[k];
                if (teth) s->rtether[q] = s->rtether[q] + s->domain[k];
            }
        }
}

/* ------------------------------------------------------------------------ */
/* record (simulation_record.f90:1205-1314)                                  */
/* ------------------------------------------------------------------------ */

void orc_evaluate_macroscopic_properties(orc *s)
{
    double vsum = 0.0, mv2sum = 0.0, pes = 0.0, vir = 0.0;
    for (int n = 0; n < s->np; n++) pes = pes + s->potenergymol[n];
    for (int n = 0; n < s->np; n++)
        for (int k = 0; k < 3; k++) {
            size_t q = 3 * (size_t)n + k;
            double vel = s->v[q];
            if (s->integration_algorithm == 0) vel = s->v[q] + 0.5 * s->a[q] * s->delta_t;
            double m = mass_of(s, n + 1);
            vsum = vsum + m * vel;
            mv2sum = mv2sum + m * (vel * vel);
        }
    for (int n = 0; n < s->np; n++) vir = vir + s->virialmol[n];
    double gnp = (double)s->globalnp;
    s->vsum = vsum; s->mv2sum = mv2sum; s->potenergysum = pes; s->virial = vir;
    s->kinenergy = (0.5 * mv2sum) / gnp;
    s->potenergy = (0.5 * pes) / gnp + s->potential_sLRC;
    s->totenergy = s->kinenergy + s->potenergy;
    s->temperature = mv2sum / (3.0 * gnp);
    s->pressure = (s->density / (gnp * 3.0)) * (mv2sum + vir / 2.0) + s->pressure_sLRC;
}

/* ------------------------------------------------------------------------ */
/* driver (md.f90 setup_MD and md_advance_vv)                                */
/* ------------------------------------------------------------------------ */

/* setup: assign_to_cell, messenger_updateborders(1), assign_to_neighbourlist,
 * then the initial force + record (setup_initial_record.f90:88-89). */
int orc_setup(orc *s)
{
    int rc;
    orc_linklist_deallocateall(s);
    if (s->force_list != 0) {
        if ((rc = orc_assign_to_cell(s))) return rc;
        if ((rc = orc_updateborders(s, 1))) return rc;
        if ((rc = orc_assign_to_neighbourlist(s))) return rc;
    }
    if ((rc = orc_compute_forces(s))) return rc;
    if ((s->iter % s->tplot) == 0) orc_evaluate_macroscopic_properties(s);
    return ORC_OK;
}

/* rebuild sequence (md.f90:150-157) with sort_mols disabled (SORT_FLAG 0). */
int orc_rebuild(orc *s)
{
    int rc;
    orc_linklist_deallocateall(s);
    orc_sendmols(s);
    if (s->force_list == 0) return ORC_OK;
    if ((rc = orc_assign_to_cell(s))) return rc;
    if ((rc = orc_updateborders(s, 1))) return rc;
    return orc_assign_to_neighbourlist(s);
}

void orc_cumulative_pressure(orc *s);

/* md_advance_vv (md.f90:143-163) for nsteps iterations; the record callback
 * is replaced by storing the macroscopic properties of every tplot step into
 * rec_out (9 doubles per record, see orc_macro) when non-null. */
int orc_run_vv(orc *s, int nsteps, double *rec_out, int rec_cap, int *nrec)
{
    int rc;
    *nrec = 0;
    for (int st = 0; st < nsteps; st++) {
        s->iter += 1;
        orc_move_vv(s, 1);
        if (s->force_list != 0 && (rc = orc_updateborders(s, 0))) return rc;
        int rebuild = orc_checkrebuild(s);
        if (rebuild && (rc = orc_rebuild(s))) return rc;
        if ((rc = orc_compute_forces(s))) return rc;
        orc_move_vv(s, 2);
        if ((s->iter % s->tplot) == 0) {
            orc_evaluate_macroscopic_properties(s);
            if (s->pressure_outflag == 1) orc_cumulative_pressure(s);
            if (rec_out && *nrec < rec_cap) {
                double *o = &rec_out[10 * (size_t)(*nrec)];
                o[0] = (double)s->iter;
                orc_macro(s, o + 1);
            }
            (*nrec)++;
        }
    }
    return ORC_OK;
}

/* Mie_potential 1: the caller's lookup tables (ntypes x ntypes, (i,j) at
 * [(i-1) + ntypes*(j-1)]) and moltype per molecule. */
int orc_set_mie(orc *s, int ntypes, const double *mass, const double *eps, const double *lr, const double *la,
                const double *C, const double *alpha, const double *shift, const double *k, const double *r0,
                const int *moltype)
{
    if (ntypes < 1 || ntypes > MIET) return ORC_ERR_PARAM;
    if (!s->moltype) s->moltype = (int *)xcalloc((size_t)s->np, sizeof(int));
    for (int n = 0; n < s->np; n++) {
        if (moltype[n] < 1 || moltype[n] > ntypes) return ORC_ERR_PARAM;
        s->moltype[n] = moltype[n];
    }
    for (int a = 0; a < ntypes; a++) {
        s->mie_mass[a] = mass[a];
        for (int b = 0; b < ntypes; b++) {
            int q = a + ntypes * b, t = a + MIET * b;
            s->mie_eps[t] = eps[q]; s->mie_lr[t] = lr[q]; s->mie_la[t] = la[q]; s->mie_C[t] = C[q];
            s->mie_alpha[t] = alpha[q]; s->mie_shift[t] = shift[q]; s->mie_k[t] = k[q]; s->mie_r0[t] = r0[q];
        }
    }
    s->mie = 1;
    return ORC_OK;
}

/* Polymer metadata upload: chainID, subchainID, funcy, bin_bflag(4). */
void orc_set_monomers(orc *s, const int *chain, const int *subchain, const int *funcy, const int *bflag)
{
    for (int n = 0; n < s->np; n++) {
        s->chainID[n] = chain[n];
        s->subchainID[n] = subchain[n];
        s->funcy[n] = funcy[n];
        for (int b = 0; b < 4; b++) s->bflag[4 * (size_t)n + b] = bflag[4 * (size_t)n + b];
    }
}

/* ------------------------------------------------------------------------ */
/* leap-frog with tags (simulation_move_particles_lfv.f90:308-514)           */
/* ------------------------------------------------------------------------ */

void orc_set_tags(orc *s, int ensemble, const int *tag, const double *rtether, const double *slidev, double k2,
                  double k4, double k6, int nthermo, double T0, double T1)
{
    s->ensemble = ensemble;
    for (int n = 0; n < s->np; n++) {
        s->tag[n] = tag ? tag[n] : 0;
        for (int k = 0; k < 3; k++) {
            s->rtether[3 * (size_t)n + k] = rtether ? rtether[3 * (size_t)n + k] : 0.0;
            s->slidev[3 * (size_t)n + k] = slidev ? slidev[3 * (size_t)n + k] : 0.0;
        }
    }
    s->teth_k2 = k2; s->teth_k4 = k4; s->teth_k6 = k6;
    s->nthermo = nthermo;
    s->therm_T[0] = T0; s->therm_T[1] = T1;
    s->zeta[0] = s->zeta[1] = 0.0;
}

void orc_set_pressure(orc *s, int flag) { s->pressure_outflag = flag; }

static int is_thermo(int t) { return t == 4 || t == 5 || t == 7; }

static int therm_region(const orc *s, int n) /* get_therm_region (:286-300) */
{
    if (s->nthermo == 2) return s->r[3 * (size_t)n + 1] > 0.0 ? 0 : 1;
    return 0;
}

/* tether_force, polynomial form (molecular_properties.f90:833-915). */
static void tether_force(orc *s, int n)
{
    double rio[3];
    for (int k = 0; k < 3; k++) rio[k] = s->r[3 * (size_t)n + k] - s->rtether[3 * (size_t)n + k];
    double mag = sqrt(rio[0] * rio[0] + rio[1] * rio[1] + rio[2] * rio[2]);
    double acct = -2.0 * s->teth_k2 * mag - 4.0 * s->teth_k4 * (mag * mag) - 6.0 * s->teth_k6 * pow(mag, 4.0);
    for (int k = 0; k < 3; k++) {
        s->a[3 * (size_t)n + k] = s->a[3 * (size_t)n + k] + acct * rio[k];
        s->rtether[3 * (size_t)n + k] = s->rtether[3 * (size_t)n + k] + s->slidev[3 * (size_t)n + k] * s->delta_t;
    }
}

void orc_move_lfv_tag(orc *s)
{
    const double dt = s->delta_t;
    double ascale[2] = {1.0, 1.0}, bscale[2] = {1.0, 1.0};
    if (s->nthermo > 0) { /* Nose-Hoover on the thermostatted tags (:325-372) */
        double mv2sum[2] = {0.0, 0.0}, tnp[2] = {0.0, 0.0};
        for (int n = 0; n < s->np; n++) {
            if (!is_thermo(s->tag[n])) continue;
            double vel[3];
            for (int k = 0; k < 3; k++) vel[k] = s->v[3 * (size_t)n + k] + 0.5 * s->a[3 * (size_t)n + k] * dt;
            int tr = therm_region(s, n);
            double d2 = 0.0;
            d2 = d2 + vel[0] * vel[0]; d2 = d2 + vel[1] * vel[1]; d2 = d2 + vel[2] * vel[2];
            mv2sum[tr] = mv2sum[tr] + 1.0 * d2;
            tnp[tr] = tnp[tr] + 1.0;
        }
        for (int r = 0; r < s->nthermo; r++) {
            double Q = 1.0 * tnp[r] * dt;
            double dz = tnp[r] > 0.0 ? (mv2sum[r] - (3.0 * tnp[r] + 1) * s->therm_T[r]) / Q : 0.0;
            s->zeta[r] = s->zeta[r] + dt * dz;
            bscale[r] = 1.0 / (1.0 + 0.5 * dt * s->zeta[r]);
            ascale[r] = (1.0 - 0.5 * dt * s->zeta[r]) * bscale[r];
        }
    }
    for (int n = 0; n < s->np; n++) {
        double *r = &s->r[3 * (size_t)n], *v = &s->v[3 * (size_t)n], *a = &s->a[3 * (size_t)n];
        const double *sv = &s->slidev[3 * (size_t)n];
        int t = s->tag[n];
        int tr;
        switch (t) {
        case 0: /* free */
            for (int k = 0; k < 3; k++) { v[k] = v[k] + dt * a[k]; r[k] = r[k] + dt * v[k]; }
            break;
        case 1: break; /* fixed */
        case 2: for (int k = 0; k < 3; k++) r[k] = r[k] + dt * sv[k]; break;
        case 3:
            tether_force(s, n);
            for (int k = 0; k < 3; k++) { v[k] = v[k] + dt * a[k]; r[k] = r[k] + dt * v[k]; }
            break;
        case 4:
            tr = therm_region(s, n);
            for (int k = 0; k < 3; k++) { v[k] = v[k] * ascale[tr] + a[k] * dt * bscale[tr]; r[k] = r[k] + v[k] * dt; }
            break;
        case 5:
            tr = therm_region(s, n);
            tether_force(s, n);
            for (int k = 0; k < 3; k++) { v[k] = v[k] * ascale[tr] + a[k] * dt * bscale[tr]; r[k] = r[k] + v[k] * dt; }
            break;
        case 6:
            tether_force(s, n);
            for (int k = 0; k < 3; k++) { v[k] = v[k] + dt * a[k]; r[k] = r[k] + dt * v[k] + dt * sv[k]; }
            break;
        case 7:
            tr = therm_region(s, n);
            tether_force(s, n);
            for (int k = 0; k < 3; k++) {
                v[k] = v[k] * ascale[tr] + a[k] * dt * bscale[tr];
                r[k] = r[k] + v[k] * dt + sv[k] * dt;
            }
            break;
        default: break;
        }
    }
    s->simtime = s->simtime + dt;
}

/* cumulative_pressure case 1 (simulation_record.f90:3151-3220). */
void orc_cumulative_pressure(orc *s)
{
    double P[9] = {0};
    double volume = s->domain[0] * s->domain[1] * s->domain[2];
    for (int n = 0; n < s->np; n++) {
        double vel[3];
        for (int k = 0; k < 3; k++) {
            vel[k] = s->v[3 * (size_t)n + k];
            if (s->integration_algorithm == 0) vel[k] = s->v[3 * (size_t)n + k] + 0.5 * s->a[3 * (size_t)n + k] * s->delta_t;
        }
        const double *rf = &s->rfmol[9 * (size_t)n];
        for (int j = 0; j < 3; j++)
            for (int k = 0; k < 3; k++) P[3 * k + j] += vel[k] * vel[j] + rf[3 * k + j] / 2.0;
    }
    for (int q = 0; q < 9; q++) s->Pxy[q] += P[q] / volume;
    s->nstress += 1;
}

void orc_pressure_average(orc *s, double out[9], int *nsamples)
{
    for (int q = 0; q < 9; q++) out[q] = s->nstress ? s->Pxy[q] / s->nstress : 0.0;
    *nsamples = s->nstress;
}

/* md_advance_lfv (md.f90:109-139) for nsteps iterations. */
int orc_run_lfv(orc *s, int nsteps, double *rec_out, int rec_cap, int *nrec)
{
    int rc;
    *nrec = 0;
    for (int st = 0; st < nsteps; st++) {
        s->iter += 1;
        if ((rc = orc_compute_forces(s))) return rc;
        if ((s->iter % s->tplot) == 0) {
            orc_evaluate_macroscopic_properties(s);
            if (s->pressure_outflag == 1) orc_cumulative_pressure(s);
            if (rec_out && *nrec < rec_cap) {
                double *o = &rec_out[10 * (size_t)(*nrec)];
                o[0] = (double)s->iter;
                orc_macro(s, o + 1);
            }
            (*nrec)++;
        }
        if (s->ensemble == 6) orc_move_lfv_tag(s);
        else orc_move_lfv(s);
        if (s->force_list != 0 && (rc = orc_updateborders(s, 0))) return rc;
        int rebuild = orc_checkrebuild(s);
        if (rebuild && st < nsteps - 1 && (rc = orc_rebuild(s))) return rc;
    }
    return ORC_OK;
}

/* Bonds found at the last list build as (owner, partner source, image code)
 * with glob_no identities; code as in orc_pair_list. */
long orc_bond_list(orc *s, int *owner, int *partner, int *code, long cap)
{
    long n = 0;
    for (int i = 1; i <= s->np; i++)
        for (int b = 0; b < s->bondcount[i - 1]; b++) {
            int j = s->bond[(size_t)(i - 1) * s->max_funcy + b];
            if (j == 0) continue;
            if (n < cap) {
                owner[n] = s->glob_no[i - 1];
                if (j <= s->np) { partner[n] = s->glob_no[j - 1]; code[n] = 13; }
                else {
                    const signed char *sh = &s->halo_shift[3 * (size_t)(j - 1)];
                    partner[n] = s->glob_no[s->halo_src[j - 1] - 1];
                    code[n] = (sh[0] + 1) + 3 * (sh[1] + 1) + 9 * (sh[2] + 1);
                }
            }
            n++;
        }
    return n;
}

/* ---- sort_mols ----------------------------------------------------------- */

/* hilbert3 of build_hilbert (functions_lib.f90:2609-2637) as the reference
 * writes it: level n is eight copies of level n-1, the k-th copy mapped by the
 * k-th entry of the array constructors for x, y and z.  Returns the point
 * count (8^n), or 0 when allocation fails. */
static size_t orc_hilbert3(int n, double **x, double **y, double **z)
{
    if (n <= 0) {
        *x = calloc(1, sizeof(double)); *y = calloc(1, sizeof(double)); *z = calloc(1, sizeof(double));
        if (!*x || !*y || !*z) return 0;
        return 1;
    }
    double *xo, *yo, *zo;
    size_t m = orc_hilbert3(n - 1, &xo, &yo, &zo);
    if (!m) return 0;
    *x = malloc(8 * m * sizeof(double)); *y = malloc(8 * m * sizeof(double)); *z = malloc(8 * m * sizeof(double));
    if (!*x || !*y || !*z) { free(xo); free(yo); free(zo); return 0; }
    double *X = *x, *Y = *y, *Z = *z;
    for (size_t i = 0; i < m; i++) {
        /* x = 0.5*(/ .5+zo, .5+yo, -.5+yo, -.5-xo, -.5-xo, -.5-yo, .5-yo, .5+zo /) */
        X[0 * m + i] = 0.5 * (0.5 + zo[i]);  X[1 * m + i] = 0.5 * (0.5 + yo[i]);
        X[2 * m + i] = 0.5 * (-0.5 + yo[i]); X[3 * m + i] = 0.5 * (-0.5 - xo[i]);
        X[4 * m + i] = 0.5 * (-0.5 - xo[i]); X[5 * m + i] = 0.5 * (-0.5 - yo[i]);
        X[6 * m + i] = 0.5 * (0.5 - yo[i]);  X[7 * m + i] = 0.5 * (0.5 + zo[i]);
        /* y = 0.5*(/ .5+xo, .5+zo, .5+zo, .5+yo, -.5+yo, -.5-zo, -.5-zo, -.5-xo /) */
        Y[0 * m + i] = 0.5 * (0.5 + xo[i]);  Y[1 * m + i] = 0.5 * (0.5 + zo[i]);
        Y[2 * m + i] = 0.5 * (0.5 + zo[i]);  Y[3 * m + i] = 0.5 * (0.5 + yo[i]);
        Y[4 * m + i] = 0.5 * (-0.5 + yo[i]); Y[5 * m + i] = 0.5 * (-0.5 - zo[i]);
        Y[6 * m + i] = 0.5 * (-0.5 - zo[i]); Y[7 * m + i] = 0.5 * (-0.5 - xo[i]);
        /* z = 0.5*(/ .5+yo, -.5+xo, -.5+xo, .5-zo, .5-zo, -.5+xo, -.5+xo, .5-yo /) */
        Z[0 * m + i] = 0.5 * (0.5 + yo[i]);  Z[1 * m + i] = 0.5 * (-0.5 + xo[i]);
        Z[2 * m + i] = 0.5 * (-0.5 + xo[i]); Z[3 * m + i] = 0.5 * (0.5 - zo[i]);
        Z[4 * m + i] = 0.5 * (0.5 - zo[i]);  Z[5 * m + i] = 0.5 * (-0.5 + xo[i]);
        Z[6 * m + i] = 0.5 * (-0.5 + xo[i]); Z[7 * m + i] = 0.5 * (0.5 - yo[i]);
    }
    free(xo); free(yo); free(zo);
    return 8 * m;
}

/* Hcurve (setup_set_parameters.f90:1140-1163): sort_flag 1 numbers the
 * blocks x fastest; sort_flag 2 is build_hilbert (functions_lib.f90:
 * 2555-2604).  hc holds nb[0]*nb[1]*nb[2] values, x fastest.  Returns
 * ORC_OK, ORC_ERR_PARAM (bad flag, a cell the curve missed, or more than 8
 * levels) or ORC_ERR_ALLOC. */
int orc_sort_table(int sort_flag, const int nb[3], int *hc)
{
    const long blocks = (long)nb[0] * nb[1] * nb[2];
    if (sort_flag == 1) {
        for (int k = 1; k <= nb[2]; k++)
            for (int j = 1; j <= nb[1]; j++)
                for (int i = 1; i <= nb[0]; i++)
                    hc[(i - 1) + nb[0] * ((j - 1) + nb[1] * (k - 1))] = i + nb[0] * (j - 1) + nb[0] * nb[1] * (k - 1);
        return ORC_OK;
    }
    if (sort_flag != 2) return ORC_ERR_PARAM;
    int maxcells = nb[0];
    if (nb[1] > maxcells) maxcells = nb[1];
    if (nb[2] > maxcells) maxcells = nb[2];
    int hindex = (int)ceil(log((double)maxcells) / log(2.0));
    if (hindex > 8) return ORC_ERR_PARAM;
    double *x, *y, *z;
    size_t n = orc_hilbert3(hindex, &x, &y, &z);
    if (!n) return ORC_ERR_ALLOC;
    if (hindex - log((double)maxcells) / log(2.0) > 0.0001) maxcells = (int)ceil(pow(8.0, (double)hindex / 3.0));
    double mn = x[0];
    for (size_t i = 0; i < n; i++) {
        if (x[i] < mn) mn = x[i];
        if (y[i] < mn) mn = y[i];
        if (z[i] < mn) mn = z[i];
    }
    const double shift = 0.00001 - mn;
    for (long b = 0; b < blocks; b++) hc[b] = -666;
    int m = 0;
    for (size_t i = 0; i < n; i++) {
        int icell = (int)ceil((x[i] + shift) * maxcells);
        int jcell = (int)ceil((y[i] + shift) * maxcells);
        int kcell = (int)ceil((z[i] + shift) * maxcells);
        if (icell <= nb[0] && jcell <= nb[1] && kcell <= nb[2]) {
            m = m + 1;
            hc[(icell - 1) + nb[0] * ((jcell - 1) + nb[1] * (kcell - 1))] = m;
        }
    }
    free(x); free(y); free(z);
    for (long b = 0; b < blocks; b++)
        if (hc[b] == -666) return ORC_ERR_PARAM;
    return ORC_OK;
}

/* The save variables of sort_mols (linklist.f90:2758-2762). */
typedef struct orc_sort_state {
    int nrebuilds;  /* starts at 1 */
    int sf2;        /* starts at 5 */
    double sf1;     /* starts at 1.5 */
} orc_sort_state;

/* sort_mols (linklist.f90:2744-2869) on np molecules: r and v are (3, np)
 * column-major and re-ordered in place, with glob (may be NULL) moved like
 * tag.  hc is the table of orc_sort_table for the block grid nblocks =
 * ceiling(domain / (sortblocksize * cellsidelength)).  *did is 0 when the
 * rebuild counter or sort_flag 0 leaves the order alone, 1 when the molecules
 * were sorted (perm[p] = old 0-based index of the molecule now at p) and 2
 * when a block overflowed ave_molperblock (order unchanged, safety factors
 * grown).  The reference's error_abort for polymers and Mie is the caller's
 * business. */
int orc_sort_mols(int np, double *r, double *v, int *glob, const double domain[3],
                  const double cellsidelength[3], int sort_flag, int sort_freq, int sortblocksize,
                  const int *hc, orc_sort_state *st, int *perm, int *did)
{
    *did = 0;
    if (st->nrebuilds != sort_freq) {
        st->nrebuilds = st->nrebuilds + 1;
        return ORC_OK;
    }
    st->nrebuilds = 1;
    if (sort_flag == 0) return ORC_OK;
    if (sort_flag != 1 && sort_flag != 2) return ORC_ERR_PARAM;
    double blocksidelength[3], halfdomain[3];
    int nblocks[3];
    for (int k = 0; k < 3; k++) {
        blocksidelength[k] = sortblocksize * cellsidelength[k];
        nblocks[k] = (int)ceil(domain[k] / blocksidelength[k]);
        halfdomain[k] = 0.5 * domain[k];
    }
    const int blocks = nblocks[0] * nblocks[1] * nblocks[2];
    int ave_molperblock = np / blocks;
    ave_molperblock = (int)ceil(ave_molperblock * st->sf1 + st->sf2);
    int *molperblock = calloc((size_t)blocks, sizeof(int));
    int *blockof = malloc((size_t)(np > 0 ? np : 1) * sizeof(int));
    if (!molperblock || !blockof) { free(molperblock); free(blockof); return ORC_ERR_ALLOC; }
    for (int n = 0; n < np; n++) {
        int ib[3];
        for (int k = 0; k < 3; k++) ib[k] = (int)ceil((r[3 * (size_t)n + k] + halfdomain[k]) / blocksidelength[k]);
        long lin = (ib[0] - 1) + (long)nblocks[0] * ((ib[1] - 1) + (long)nblocks[1] * (ib[2] - 1));
        if (lin < 0) lin = 0;  /* a molecule on the lower face: see the CUDA path */
        if (lin > blocks - 1) lin = blocks - 1;
        int i = hc[lin];
        molperblock[i - 1] = molperblock[i - 1] + 1;
        if (molperblock[i - 1] > ave_molperblock) {
            st->sf1 = st->sf1 + 0.1;
            st->sf2 = st->sf2 + 5;
            free(molperblock); free(blockof);
            *did = 2;
            return ORC_OK;
        }
        blockof[n] = i;
    }
    /* copy back block by block, each block in its molecules' old order */
    int *start = malloc((size_t)blocks * sizeof(int));
    double *r0 = malloc(3 * (size_t)np * sizeof(double) + 1), *v0 = malloc(3 * (size_t)np * sizeof(double) + 1);
    int *g0 = glob ? malloc((size_t)np * sizeof(int) + 1) : NULL;
    if (!start || !r0 || !v0 || (glob && !g0)) {
        free(start); free(r0); free(v0); free(g0); free(molperblock); free(blockof);
        return ORC_ERR_ALLOC;
    }
    memcpy(r0, r, 3 * (size_t)np * sizeof(double));
    memcpy(v0, v, 3 * (size_t)np * sizeof(double));
    if (glob) memcpy(g0, glob, (size_t)np * sizeof(int));
    int pos = 0;
    for (int b = 0; b < blocks; b++) { start[b] = pos; pos += molperblock[b]; }
    for (int n = 0; n < np; n++) {
        int p = start[blockof[n] - 1]++;
        perm[p] = n;
        for (int k = 0; k < 3; k++) {
            r[3 * (size_t)p + k] = r0[3 * (size_t)n + k];
            v[3 * (size_t)p + k] = v0[3 * (size_t)n + k];
        }
        if (glob) glob[p] = g0[n];
    }
    free(start); free(r0); free(v0); free(g0); free(molperblock); free(blockof);
    *did = 1;
    return ORC_OK;
}
