/*
 * CPU restatement of Mjolnir's per-step hot path.  TEST INFRASTRUCTURE ONLY:
 * see oracle.h.  Compiled with -ffp-contract=off so that every product and sum
 * rounds the way the reference's (non -Ofast) build does; the expressions keep
 * the reference's operation order so that forces, lists and noise-free
 * trajectories can be compared with the reference bit for bit.
 */
#include "oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ units */

/* core/Unit.hpp:23-26 (SI defaults) + core/Unit.hpp:150-156 (eps0 in e^2) +
 * input/read_units.hpp:32-49 (kcal/mol) + :73-91 (angstrom). */
void orc_units(double* kB, double* NA, double* eps0, double* L_to_volume)
{
    const double boltzmann   = 1.38064852e-23;
    const double avogadro    = 6.022140857e23;
    const double e_charge    = 1.6021766208e-19;
    const double vacuum_perm = 8.854187817e-12;
    const double J_to_cal    = 1.0 / 4.184;
    const double m_to_ang    = 1e+10;

    double kb  = boltzmann;
    double eps = (vacuum_perm / e_charge) / e_charge;
    kb  = kb * (J_to_cal / 1000.0) * avogadro;
    eps = eps * (1000.0 / J_to_cal) / avogadro;
    eps = eps / m_to_ang;
    if(kB)          {*kB = kb;}
    if(NA)          {*NA = avogadro;}
    if(eps0)        {*eps0 = eps;}
    if(L_to_volume) {*L_to_volume = 1e-3 * pow(m_to_ang, 3);}
}

/* forcefield/global/DebyeHuckelPotential.hpp:126-174 */
void orc_dh_params(double T, double c, double cutoff_ratio, double out[5])
{
    double kB, NA, eps0, L2V;
    orc_units(&kB, &NA, &eps0, &L2V);
    const double pi   = 3.14159265358979323846264338;
    const double epsk = (249.4 - 0.788 * T + 7.2e-4 * T * T) *
                        (1. - 2.551e-1 * c + 5.151e-2 * c * c - 6.889e-3 * c * c * c);
    const double inv_4pi = 1.0 / (4 * pi * eps0 * epsk);
    const double I       = c / L2V;
    const double debye   = sqrt((eps0 * epsk * kB * T) / (2 * NA * I));
    const double inv_debye = 1. / debye;
    out[0] = debye;
    out[1] = inv_debye;
    out[2] = cutoff_ratio * debye;
    out[3] = exp(-cutoff_ratio) / (debye * cutoff_ratio);
    out[4] = inv_4pi;
}

/* ------------------------------------------------------------------ state */

typedef struct
{
    int     on;
    int64_t np;          /* participants, in input order                    */
    int64_t* idx;
    double*  p0;         /* radius / charge / sigma per participant index   */
    double*  p1;         /* LJ epsilon                                      */
    double*  pp0;        /* per-particle copies (0 for non-participants)    */
    double*  pp1;
    char*    is_part;    /* per particle                                    */
    char*    is_lead;    /* per particle: participant but not the last one  */
    double   cutoff;     /* max_cutoff_length                               */
    double   margin;
    double   current_margin;
    /* potential constants */
    double   eps, cutoff_ratio, coef_at_cutoff;
    double   dh[5];
    int      kind;       /* first term: ORC_EXV ...; third term: ORC_LJ ...           */
    int      power;      /* InversePower n                                            */
    /* current half list: partners of particle i are nbr[lb[i] .. le[i]) */
    int64_t* lb;
    int64_t* le;
    int64_t* nbr;
    int64_t  nnbr;
    int64_t  rebuilds;
} orc_global;

struct orc_state
{
    orc_spec s;          /* array pointers below are private copies         */
    int64_t  n;
    double  *pos, *vel, *force, *mass, *rmass, *gamma;
    double   lower[3], upper[3], width[3], halfw[3];
    int64_t *mol;
    int64_t *ex_ranges, *ex_idx;
    orc_global g[3];
    /* integrator */
    double   dt, halfdt, kB, T;
    double  *exp_gamma_dt, *noise_coeff;
    double  *accel;      /* UnderdampedLangevin: [3n] acceleration with noise */
    double  *gjf_b;      /* G-JF: [n] b = 1 / (1 + alpha dt / 2m)              */
    uint64_t step;
    /* local terms */
    int64_t  nbond, nangle, ndihd;
    int64_t *bond_idx, *angle_idx, *dihd_idx;
    double  *bond_k, *bond_v0, *angle_k, *angle_v0, *dihd_k, *dihd_v0;
    int32_t *dihd_n;
};

static void* dup(const void* p, size_t bytes)
{
    if(!p || bytes == 0) {return NULL;}
    void* q = malloc(bytes);
    memcpy(q, p, bytes);
    return q;
}

/* core/BoundaryCondition.hpp:81-91 (periodic) and :24-27 (unlimited) */
static inline void adjust_direction(const orc_state* st, const double* from,
                                    const double* to, double* dr)
{
    for(int k=0; k<3; ++k)
    {
        double d = to[k] - from[k];
        if(st->s.boundary == ORC_PERIODIC)
        {
            if     (d < -st->halfw[k]) {d += st->width[k];}
            else if(d >=  st->halfw[k]) {d -= st->width[k];}
        }
        dr[k] = d;
    }
}
/* core/BoundaryCondition.hpp:93-102 */
static inline void adjust_position(const orc_state* st, double* p)
{
    if(st->s.boundary != ORC_PERIODIC) {return;}
    for(int k=0; k<3; ++k)
    {
        if     (p[k] <  st->lower[k]) {p[k] += st->width[k];}
        else if(p[k] >= st->upper[k]) {p[k] -= st->width[k];}
    }
}
/* math/Vector.hpp:84-88 */
static inline double length_sq(const double* v)
{
    return v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
}

/* ------------------------------------------------------------- topology */

typedef struct {int64_t* off; int64_t* adj;} graph;

static graph bond_graph(const orc_state* st)
{
    /* edges of connection kind "bond": BondLength (topology "bond",
     * BondLengthInteraction.hpp write_topology) and the Dummy chain */
    const int64_t n = st->n;
    int64_t nb = st->nbond + ((st->s.single_molecule && n > 1) ? n - 1 : 0);
    int64_t* a = malloc(sizeof(int64_t) * 2 * (nb ? nb : 1));
    int64_t k = 0;
    for(int64_t b=0; b<st->nbond; ++b)
    {
        a[2*k] = st->bond_idx[2*b]; a[2*k+1] = st->bond_idx[2*b+1]; ++k;
    }
    if(st->s.single_molecule) {for(int64_t i=0; i+1<n; ++i) {a[2*k] = i; a[2*k+1] = i+1; ++k;}}
    graph g;
    g.off = calloc((size_t)n + 1, sizeof(int64_t));
    for(int64_t e=0; e<k; ++e) {g.off[a[2*e]+1]++; g.off[a[2*e+1]+1]++;}
    for(int64_t i=0; i<n; ++i) {g.off[i+1] += g.off[i];}
    int64_t* fill = calloc((size_t)n, sizeof(int64_t));
    g.adj = malloc(sizeof(int64_t) * (2 * k + 1));
    /* Topology::add_connection appends each new edge to both adjacency lists
     * in the order the edges are added (core/Topology.hpp:165-195). */
    for(int64_t e=0; e<k; ++e)
    {
        const int64_t i = a[2*e], j = a[2*e+1];
        /* add_connection skips an edge that is already present */
        int dupe = 0;
        for(int64_t q=g.off[i]; q<g.off[i]+fill[i]; ++q) {if(g.adj[q] == j) {dupe = 1; break;}}
        if(dupe) {continue;}
        g.adj[g.off[i] + fill[i]++] = j;
        if(i != j) {g.adj[g.off[j] + fill[j]++] = i;}
    }
    /* compact (duplicates leave holes) */
    int64_t w = 0, prev = 0;
    for(int64_t i=0; i<n; ++i)
    {
        const int64_t b = prev, e = g.off[i] + fill[i];
        prev = g.off[i+1];
        g.off[i] = w;
        for(int64_t q=b; q<e; ++q) {g.adj[w++] = g.adj[q];}
    }
    g.off[n] = w;
    free(fill); free(a);
    return g;
}

/* core/Topology.hpp:280-316: one pass in particle order; a particle takes the
 * molecule id of its first "bond" neighbour that already has one. */
static void construct_molecules(orc_state* st, const graph* g)
{
    const int64_t n = st->n;
    int64_t next = 0;
    for(int64_t i=0; i<n; ++i) {st->mol[i] = -1;}
    for(int64_t i=0; i<n; ++i)
    {
        for(int64_t q=g->off[i]; q<g->off[i+1]; ++q)
        {
            if(st->mol[g->adj[q]] != -1) {st->mol[i] = st->mol[g->adj[q]]; break;}
        }
        if(st->mol[i] == -1) {st->mol[i] = next++;}
    }
}

static int cmp_i64(const void* a, const void* b)
{
    const int64_t x = *(const int64_t*)a, y = *(const int64_t*)b;
    return (x > y) - (x < y);
}

/* core/Topology.hpp:243-260 list_adjacent_within + core/ExclusionList.hpp:207-232:
 * i itself and every particle within `dist` "bond" edges, sorted, unique. */
static void build_exclusions(orc_state* st, const graph* g)
{
    const int64_t n = st->n;
    const int dist = st->s.ignore_bond_within;
    st->ex_ranges = malloc(sizeof(int64_t) * ((size_t)n + 1));
    int64_t cap = n * 4 + 16, used = 0;
    st->ex_idx = malloc(sizeof(int64_t) * (size_t)cap);
    int64_t* buf = malloc(sizeof(int64_t) * 64);
    int64_t bcap = 64;
    int64_t* front = malloc(sizeof(int64_t) * 64);
    int64_t fcap = 64;
    for(int64_t i=0; i<n; ++i)
    {
        int64_t nb = 0;
        buf[nb++] = i;
        /* breadth-first expansion gives the same set as the recursive walk */
        int64_t fb = 0, fe = 0;
        if(dist > 0)
        {
            front[fe++] = i;
            for(int d=0; d<dist; ++d)
            {
                const int64_t lb = fb, le = fe;
                for(int64_t f=lb; f<le; ++f)
                {
                    const int64_t u = front[f];
                    for(int64_t q=g->off[u]; q<g->off[u+1]; ++q)
                    {
                        if(nb == bcap) {bcap *= 2; buf = realloc(buf, sizeof(int64_t) * bcap);}
                        buf[nb++] = g->adj[q];
                        if(fe == fcap) {fcap *= 2; front = realloc(front, sizeof(int64_t) * fcap);}
                        front[fe++] = g->adj[q];
                    }
                }
                fb = le;
            }
        }
        qsort(buf, (size_t)nb, sizeof(int64_t), cmp_i64);
        int64_t u = 0;
        for(int64_t q=0; q<nb; ++q) {if(q == 0 || buf[q] != buf[u-1]) {buf[u++] = buf[q];}}
        st->ex_ranges[i] = used;
        if(used + u > cap) {while(used + u > cap) {cap *= 2;} st->ex_idx = realloc(st->ex_idx, sizeof(int64_t) * cap);}
        memcpy(st->ex_idx + used, buf, sizeof(int64_t) * (size_t)u);
        used += u;
    }
    st->ex_ranges[n] = used;
    free(buf); free(front);
}

/* core/ExclusionList.hpp:56-84 (groups are all "NONE" with no group rule) */
static inline int is_excluded(const orc_state* st, int64_t i, int64_t j)
{
    if(st->s.ignore_molecule == ORC_IGNORE_SELF   && st->mol[i] == st->mol[j]) {return 1;}
    if(st->s.ignore_molecule == ORC_IGNORE_OTHERS && st->mol[i] != st->mol[j]) {return 1;}
    for(int64_t q=st->ex_ranges[i]; q<st->ex_ranges[i+1]; ++q)
    {
        if(st->ex_idx[q] >  j) {break;}
        if(st->ex_idx[q] == j) {return 1;}
    }
    return 0;
}

/* ------------------------------------------------------------- create */

static void setup_global(orc_state* st, int gi, int on, int64_t np, const int64_t* idx,
                         const double* p0, const double* p1, double cutoff_ratio, double margin)
{
    orc_global* g = &st->g[gi];
    memset(g, 0, sizeof(*g));
    g->on = on;
    if(!on) {return;}
    const int64_t n = st->n;
    g->np  = np;
    g->idx = dup(idx, sizeof(int64_t) * np);
    g->p0  = dup(p0, sizeof(double) * np);
    g->p1  = p1 ? dup(p1, sizeof(double) * np) : NULL;
    g->pp0 = calloc((size_t)n, sizeof(double));
    g->pp1 = calloc((size_t)n, sizeof(double));
    g->is_part = calloc((size_t)n, 1);
    g->is_lead = calloc((size_t)n, 1);
    for(int64_t k=0; k<np; ++k)
    {
        g->pp0[idx[k]] = p0[k];
        if(p1) {g->pp1[idx[k]] = p1[k];}
        g->is_part[idx[k]] = 1;
        if(k + 1 < np) {g->is_lead[idx[k]] = 1;}   /* ParameterList leading_participants */
    }
    g->margin       = margin;
    g->cutoff_ratio = cutoff_ratio;
    g->lb = calloc((size_t)n, sizeof(int64_t));
    g->le = calloc((size_t)n, sizeof(int64_t));
    if(gi == 0)        /* ExcludedVolumePotential.hpp:44-48, :92-106 and the family */
    {
        g->kind = st->s.exv_kind;
        g->power = st->s.exv_power;
        /* InversePowerPotential.hpp:32-36: (1/rc)^n; the others (1/rc)^12 */
        g->coef_at_cutoff = g->kind == ORC_INVERSE_POWER ? pow(1.0 / cutoff_ratio, g->power)
                                                        : pow(1.0 / cutoff_ratio, 12);
        double mr = 0, mc = 0;
        for(int64_t k=0; k<np; ++k) {if(mr < p0[k]) {mr = p0[k];}}
        if(g->kind == ORC_HARD_CORE_EXV)
        {
            for(int64_t k=0; k<np; ++k) {if(mc < p1[k]) {mc = p1[k];}}
            /* HardCoreExcludedVolumePotential.hpp:109-126 */
            g->cutoff = np == 0 ? 1.0 : mr * 2 * cutoff_ratio + mc * 2;
        }
        else
        {
            g->cutoff = np == 0 ? 1.0 : mr * 2 * cutoff_ratio;
        }
    }
    else if(gi == 1)   /* DebyeHuckelPotential.hpp:126-167, :245-248 */
    {
        orc_dh_params(st->s.temperature, st->s.ionic_strength, cutoff_ratio, g->dh);
        g->cutoff = g->dh[0] * cutoff_ratio;
    }
    else               /* LennardJonesPotential.hpp:36-41, :75-91 and the family */
    {
        g->kind = st->s.lj_kind;
        /* WCAPotential.hpp: no shift; the others: LennardJones' shift */
        g->coef_at_cutoff = g->kind == ORC_WCA ? 0.0 :
                            pow(1.0 / cutoff_ratio, 12) - pow(1.0 / cutoff_ratio, 6);
        double ms = 0;
        for(int64_t k=0; k<np; ++k) {if(ms < p0[k]) {ms = p0[k];}}
        g->cutoff = np == 0 ? 1.0 : ms * cutoff_ratio;
    }
}

static void make_list(orc_state* st, int gi);

orc_state* orc_create(const orc_spec* s)
{
    if(!s || s->n <= 0) {return NULL;}
    orc_state* st = calloc(1, sizeof(orc_state));
    st->s = *s;
    const int64_t n = s->n;
    st->n = n;
    st->pos   = dup(s->pos, sizeof(double) * 3 * n);
    st->vel   = s->vel ? dup(s->vel, sizeof(double) * 3 * n) : calloc(3 * (size_t)n, sizeof(double));
    st->force = calloc(3 * (size_t)n, sizeof(double));
    st->mass  = dup(s->mass, sizeof(double) * n);
    st->rmass = malloc(sizeof(double) * n);
    for(int64_t i=0; i<n; ++i) {st->rmass[i] = 1.0 / st->mass[i];}
    st->gamma = s->gamma ? dup(s->gamma, sizeof(double) * n) : calloc((size_t)n, sizeof(double));
    for(int k=0; k<3; ++k)
    {
        st->lower[k] = s->lower[k];
        st->upper[k] = s->upper[k];
        st->width[k] = s->upper[k] - s->lower[k];
        st->halfw[k] = st->width[k] / 2;
    }
    /* System::initialize wraps every position into the box (System.hpp:63-67) */
    for(int64_t i=0; i<n; ++i) {adjust_position(st, st->pos + 3*i);}

    st->nbond = s->nbond; st->nangle = s->nangle; st->ndihd = s->ndihd;
    st->bond_idx  = dup(s->bond_idx,  sizeof(int64_t) * 2 * s->nbond);
    st->bond_k    = dup(s->bond_k,    sizeof(double) * s->nbond);
    st->bond_v0   = dup(s->bond_v0,   sizeof(double) * s->nbond);
    st->angle_idx = dup(s->angle_idx, sizeof(int64_t) * 3 * s->nangle);
    st->angle_k   = dup(s->angle_k,   sizeof(double) * s->nangle);
    st->angle_v0  = dup(s->angle_v0,  sizeof(double) * s->nangle);
    st->dihd_idx  = dup(s->dihd_idx,  sizeof(int64_t) * 4 * s->ndihd);
    st->dihd_k    = dup(s->dihd_k,    sizeof(double) * s->ndihd);
    st->dihd_n    = dup(s->dihd_n,    sizeof(int32_t) * s->ndihd);
    st->dihd_v0   = dup(s->dihd_v0,   sizeof(double) * s->ndihd);

    st->mol = malloc(sizeof(int64_t) * n);
    graph g = bond_graph(st);
    construct_molecules(st, &g);
    build_exclusions(st, &g);
    free(g.off); free(g.adj);

    setup_global(st, 0, s->exv_on, s->exv_n, s->exv_idx, s->exv_radius,
                 s->exv_kind == ORC_HARD_CORE_EXV ? s->exv_core : NULL, s->exv_cutoff, s->exv_margin);
    setup_global(st, 1, s->dh_on,  s->dh_n,  s->dh_idx,  s->dh_charge,  NULL, s->dh_cutoff,  s->dh_margin);
    setup_global(st, 2, s->lj_on,  s->lj_n,  s->lj_idx,  s->lj_sigma,   s->lj_eps, s->lj_cutoff, s->lj_margin);
    if(s->exv_on) {st->g[0].eps = s->exv_eps;}
    for(int gi=0; gi<3; ++gi) {if(st->g[gi].on) {make_list(st, gi); st->g[gi].rebuilds = 0;}}

    orc_units(&st->kB, NULL, NULL, NULL);
    st->T = s->temperature;
    st->dt = s->dt;
    st->halfdt = s->dt / 2;
    st->exp_gamma_dt = calloc((size_t)n, sizeof(double));
    st->noise_coeff  = calloc((size_t)n, sizeof(double));
    st->accel        = calloc((size_t)(3 * n), sizeof(double));
    st->gjf_b        = calloc((size_t)n, sizeof(double));
    return st;
}

void orc_destroy(orc_state* st)
{
    if(!st) {return;}
    void* ptrs[] = {st->pos, st->vel, st->force, st->mass, st->rmass, st->gamma, st->mol,
                    st->ex_ranges, st->ex_idx, st->exp_gamma_dt, st->noise_coeff, st->accel, st->gjf_b,
                    st->bond_idx, st->bond_k, st->bond_v0, st->angle_idx, st->angle_k,
                    st->angle_v0, st->dihd_idx, st->dihd_k, st->dihd_n, st->dihd_v0};
    for(size_t k=0; k<sizeof(ptrs)/sizeof(ptrs[0]); ++k) {free(ptrs[k]);}
    for(int gi=0; gi<3; ++gi)
    {
        orc_global* g = &st->g[gi];
        free(g->idx); free(g->p0); free(g->p1); free(g->pp0); free(g->pp1);
        free(g->is_part); free(g->is_lead); free(g->lb); free(g->le); free(g->nbr);
    }
    free(st);
}

void orc_molecules(const orc_state* st, int64_t* mol)
{
    memcpy(mol, st->mol, sizeof(int64_t) * st->n);
}

int64_t orc_exclusions(const orc_state* st, int64_t* ranges, int64_t* idx, int64_t cap)
{
    const int64_t tot = st->ex_ranges[st->n];
    if(ranges) {memcpy(ranges, st->ex_ranges, sizeof(int64_t) * (st->n + 1));}
    if(idx) {memcpy(idx, st->ex_idx, sizeof(int64_t) * (tot < cap ? tot : cap));}
    return tot;
}

/* -------------------------------------------------------- neighbour list */

/* The set a cell list yields is {j : has_interaction(i, j) and
 * |adjust_direction(r_i, r_j)|^2 < (cutoff (1 + margin))^2} for every leading
 * participant i (PeriodicGridCellList.hpp:296-347; UnlimitedGridCellList.hpp
 * :198-250), partners sorted by j (:340-341).  The reference's cells are at
 * least cutoff (1 + margin) wide, so the stencil never decides membership; the
 * grid below only has to be conservative as well, and the distance test, in the
 * reference's operation order, decides. */
static int64_t half_list(const orc_state* st, int gi, const double* pos,
                         int64_t* lb, int64_t* le, int64_t** out_nbr, int64_t* out_cap)
{
    const orc_global* g = &st->g[gi];
    const int64_t n = st->n;
    const double r_c  = g->cutoff * (1. + g->margin);
    const double r_c2 = r_c * r_c;

    double lo[3], hi[3];
    int64_t dims[3];
    const int periodic = st->s.boundary == ORC_PERIODIC;
    int brute = 0;
    for(int k=0; k<3; ++k)
    {
        if(periodic) {lo[k] = st->lower[k]; hi[k] = st->upper[k];}
        else
        {
            lo[k] = 1e300; hi[k] = -1e300;
            for(int64_t q=0; q<g->np; ++q)
            {
                const double x = pos[3*g->idx[q]+k];
                if(x < lo[k]) {lo[k] = x;}
                if(x > hi[k]) {hi[k] = x;}
            }
            if(g->np == 0) {lo[k] = 0; hi[k] = 1;}
        }
        const double w = (hi[k] - lo[k]) / (r_c * (1 + 1e-9));
        dims[k] = (int64_t)floor(w);      /* cells at least r_c wide */
        if(dims[k] < 1) {dims[k] = 1;}
        if(periodic && dims[k] < 3) {brute = 1;}
        if(dims[k] > 2048) {dims[k] = 2048;}
    }
    if(brute) {dims[0] = dims[1] = dims[2] = 1;}
    const int64_t ncell = dims[0] * dims[1] * dims[2];

    const int64_t npart = g->np ? g->np : 1;
    int64_t* cell_of = malloc(sizeof(int64_t) * npart);
    int64_t* cstart  = calloc((size_t)ncell + 1, sizeof(int64_t));
    int64_t* members = malloc(sizeof(int64_t) * npart);
    double cw[3];
    for(int k=0; k<3; ++k) {cw[k] = (hi[k] - lo[k]) / (double)dims[k]; if(!(cw[k] > 0)) {cw[k] = 1;}}
    for(int64_t q=0; q<g->np; ++q)
    {
        int64_t c[3];
        for(int k=0; k<3; ++k)
        {
            int64_t v = brute ? 0 : (int64_t)floor((pos[3*g->idx[q]+k] - lo[k]) / cw[k]);
            if(v < 0) {v = 0;}
            if(v >= dims[k]) {v = dims[k] - 1;}
            c[k] = v;
        }
        cell_of[q] = c[0] + dims[0] * (c[1] + dims[1] * c[2]);
        cstart[cell_of[q] + 1]++;
    }
    for(int64_t c=0; c<ncell; ++c) {cstart[c+1] += cstart[c];}
    int64_t* fill = calloc((size_t)ncell, sizeof(int64_t));
    for(int64_t q=0; q<g->np; ++q) {members[cstart[cell_of[q]] + fill[cell_of[q]]++] = g->idx[q];}
    free(fill);

    int64_t cap = *out_cap, cnt = 0;
    int64_t* nbr = *out_nbr;
    int64_t pcap = 1024;
    int64_t* part = malloc(sizeof(int64_t) * pcap);
    for(int64_t i=0; i<n; ++i) {lb[i] = le[i] = 0;}

    for(int64_t q=0; q+1<g->np; ++q)            /* leading participants */
    {
        const int64_t i = g->idx[q];
        const double* ri = pos + 3*i;
        int64_t np_ = 0;
        const int64_t cid = cell_of[q];
        const int64_t cc[3] = {cid % dims[0], (cid / dims[0]) % dims[1], cid / (dims[0] * dims[1])};
        const int span = brute ? 0 : 1;
        for(int dz=-span; dz<=span; ++dz)
        for(int dy=-span; dy<=span; ++dy)
        for(int dx=-span; dx<=span; ++dx)
        {
            int64_t x = cc[0] + dx, y = cc[1] + dy, z = cc[2] + dz;
            if(periodic)
            {
                x = (x + dims[0]) % dims[0]; y = (y + dims[1]) % dims[1]; z = (z + dims[2]) % dims[2];
            }
            else if(x < 0 || y < 0 || z < 0 || x >= dims[0] || y >= dims[1] || z >= dims[2]) {continue;}
            const int64_t c = x + dims[0] * (y + dims[1] * z);
            for(int64_t m=cstart[c]; m<cstart[c+1]; ++m)
            {
                const int64_t j = members[m];
                if(!(i < j) || is_excluded(st, i, j)) {continue;}   /* has_interaction */
                double dr[3];
                adjust_direction(st, ri, pos + 3*j, dr);
                if(length_sq(dr) < r_c2)
                {
                    if(np_ == pcap) {pcap *= 2; part = realloc(part, sizeof(int64_t) * pcap);}
                    part[np_++] = j;
                }
            }
        }
        qsort(part, (size_t)np_, sizeof(int64_t), cmp_i64);
        if(cnt + np_ > cap)
        {
            while(cnt + np_ > cap) {cap = cap ? cap * 2 : 4096;}
            nbr = realloc(nbr, sizeof(int64_t) * (size_t)cap);
        }
        memcpy(nbr + cnt, part, sizeof(int64_t) * (size_t)np_);
        lb[i] = cnt;
        cnt += np_;
        le[i] = cnt;
    }
    free(part); free(cell_of); free(cstart); free(members);
    *out_nbr = nbr; *out_cap = cap;
    return cnt;
}

static void make_list(orc_state* st, int gi)
{
    orc_global* g = &st->g[gi];
    int64_t* nbr = NULL;
    int64_t  c   = 0;
    free(g->nbr);
    g->nnbr = half_list(st, gi, st->pos, g->lb, g->le, &nbr, &c);
    g->nbr = nbr;
    g->current_margin = g->cutoff * g->margin;   /* ...GridCellList::make, last line */
    g->rebuilds++;
}

int64_t orc_neighbors(const orc_state* st, int term, const double* pos,
                      int64_t* pairs, int64_t cap)
{
    const int gi = term - ORC_TERM_EXV;
    if(gi < 0 || gi > 2 || !st->g[gi].on) {return -1;}
    const orc_global* g = &st->g[gi];
    int64_t* lb = calloc((size_t)st->n, sizeof(int64_t));
    int64_t* le = calloc((size_t)st->n, sizeof(int64_t));
    int64_t* nbr = NULL; int64_t c = 0;
    const int64_t cnt = half_list(st, gi, pos ? pos : st->pos, lb, le, &nbr, &c);
    int64_t k = 0;
    for(int64_t q=0; q+1<g->np; ++q)
    {
        const int64_t i = g->idx[q];
        for(int64_t m=lb[i]; m<le[i]; ++m)
        {
            if(k < cap && pairs) {pairs[2*k] = i; pairs[2*k+1] = nbr[m];}
            ++k;
        }
    }
    free(lb); free(le); free(nbr);
    return k == cnt ? k : -2;
}

/* ---------------------------------------------------------------- forces */

/* forcefield/global/GlobalPairExcludedVolumeInteraction.hpp:148-195 */
static double exvfam_force(const orc_state* st, const orc_global* g, const double* pos,
                           double* force, int need_force);

static double exv_force(const orc_state* st, const orc_global* g, const double* pos,
                        double* force, int need_force)
{
    if(g->kind != ORC_EXV) {return exvfam_force(st, g, pos, force, need_force);}
    const double coef_at_cutoff  = g->coef_at_cutoff;
    const double cutoff_ratio    = g->cutoff_ratio;
    const double cutoff_ratio_sq = cutoff_ratio * cutoff_ratio;
    const double epsilon   = g->eps;
    const double epsilon12 = epsilon * 12;
    double energy = 0;
    for(int64_t q=0; q+1<g->np; ++q)
    {
        const int64_t i = g->idx[q];
        for(int64_t m=g->lb[i]; m<g->le[i]; ++m)
        {
            const int64_t j = g->nbr[m];
            const double radius = g->pp0[i] + g->pp0[j];       /* prepare_params */
            double rij[3];
            adjust_direction(st, pos + 3*i, pos + 3*j, rij);
            const double l_sq = length_sq(rij);
            const double sigma_sq = radius * radius;
            if(sigma_sq * cutoff_ratio_sq < l_sq) {continue;}
            if(need_force)
            {
                const double rcp_l_sq = 1.0 / l_sq;
                const double s2l2     = sigma_sq * rcp_l_sq;
                const double s6l6     = s2l2 * s2l2 * s2l2;
                const double coef = -epsilon12 * s6l6 * s6l6 * rcp_l_sq;
                for(int k=0; k<3; ++k)
                {
                    const double f = rij[k] * coef;
                    force[3*i+k] += f;
                    force[3*j+k] -= f;
                }
                energy += epsilon * (s6l6 * s6l6 - coef_at_cutoff);
            }
            else   /* calc_energy, :100-132 */
            {
                const double s2l2 = sigma_sq / l_sq;
                const double s6l6 = s2l2 * s2l2 * s2l2;
                energy += epsilon * (s6l6 * s6l6 - coef_at_cutoff);
            }
        }
    }
    return energy;
}

/* generic loop forcefield/global/GlobalPairInteraction.hpp:148-213 with
 * DebyeHuckelPotential::potential/derivative (DebyeHuckelPotential.hpp:44-61) */
static double dh_force(const orc_state* st, const orc_global* g, const double* pos,
                       double* force, int need_force)
{
    const double debye = g->dh[0], inv_debye = g->dh[1], abs_cutoff = g->dh[2];
    const double coef_at_cutoff = g->dh[3], inv4pi = g->dh[4];
    double energy = 0;
    for(int64_t q=0; q+1<g->np; ++q)
    {
        const int64_t i = g->idx[q];
        for(int64_t m=g->lb[i]; m<g->le[i]; ++m)
        {
            const int64_t j = g->nbr[m];
            const double qq = inv4pi * g->pp0[i] * g->pp0[j];     /* prepare_params */
            double rij[3];
            adjust_direction(st, pos + 3*i, pos + 3*j, rij);
            const double l2 = length_sq(rij);
            if(need_force)
            {
                const double rl = 1.0 / sqrt(l2);
                const double l  = l2 * rl;
                double f_mag = 0.0;
                if(!(abs_cutoff <= l))
                {
                    f_mag = -qq * (debye + l) * inv_debye / (l * l) * exp(-l * inv_debye);
                }
                if(f_mag == 0.0) {continue;}
                const double c = f_mag * rl;
                for(int k=0; k<3; ++k)
                {
                    const double f = rij[k] * c;
                    force[3*i+k] += f;
                    force[3*j+k] -= f;
                }
                energy += (abs_cutoff <= l) ? 0.0 :
                          qq * (exp(-l * inv_debye) / l - coef_at_cutoff);
            }
            else
            {
                const double l = sqrt(l2);
                energy += (abs_cutoff <= l) ? 0.0 :
                          qq * (exp(-l * inv_debye) / l - coef_at_cutoff);
            }
        }
    }
    return energy;
}

/* The ExcludedVolume family through the generic pair loop
 * (GlobalPairInteraction.hpp:148-213): InversePowerPotential
 * (InversePowerPotential.hpp:38-57, sigma_ij = r_i + r_j, :185-188) and
 * HardCoreExcludedVolumePotential (HardCoreExcludedVolumePotential.hpp:44-80,
 * sigma_ij = s_i + s_j and R_ij = c_i + c_j, :209-217). */
static double exvfam_derivative(const orc_global* g, double r, double sigma, double radius)
{
    if(g->kind == ORC_INVERSE_POWER)
    {
        if(sigma * g->cutoff_ratio < r) {return 0.0;}
        const double rinv = 1.0 / r;
        const double d_r = sigma * rinv;
        const double drn = pow(d_r, g->power);
        return -g->power * g->eps * drn * rinv;
    }
    if(sigma * g->cutoff_ratio + radius < r) {return 0.0;}
    if(r < radius) {return INFINITY;}
    const double gapinv = 1 / (r - radius);
    const double sigma1gap1 = sigma * gapinv;
    const double sigma3gap3 = sigma1gap1 * sigma1gap1 * sigma1gap1;
    const double sigma6gap6 = sigma3gap3 * sigma3gap3;
    return -12.0 * g->eps * sigma6gap6 * sigma6gap6 * gapinv;
}

static double exvfam_potential(const orc_global* g, double r, double sigma, double radius)
{
    if(g->kind == ORC_INVERSE_POWER)
    {
        if(sigma * g->cutoff_ratio < r) {return 0.0;}
        const double d_r = sigma / r;
        const double drn = pow(d_r, g->power);
        return g->eps * (drn - g->coef_at_cutoff);
    }
    if(sigma * g->cutoff_ratio + radius < r) {return 0;}
    if(r < radius) {return INFINITY;}
    const double gap = r - radius;
    const double sigma1gap1 = sigma / gap;
    const double sigma3gap3 = sigma1gap1 * sigma1gap1 * sigma1gap1;
    const double sigma6gap6 = sigma3gap3 * sigma3gap3;
    return g->eps * (sigma6gap6 * sigma6gap6 - g->coef_at_cutoff);
}

static double exvfam_force(const orc_state* st, const orc_global* g, const double* pos,
                           double* force, int need_force)
{
    double energy = 0;
    for(int64_t q=0; q+1<g->np; ++q)
    {
        const int64_t i = g->idx[q];
        for(int64_t m=g->lb[i]; m<g->le[i]; ++m)
        {
            const int64_t j = g->nbr[m];
            const double sigma  = g->pp0[i] + g->pp0[j];
            const double radius = g->kind == ORC_HARD_CORE_EXV ? g->pp1[i] + g->pp1[j] : 0.0;
            double rij[3];
            adjust_direction(st, pos + 3*i, pos + 3*j, rij);
            const double l2 = length_sq(rij);
            if(need_force)
            {
                const double rl = 1.0 / sqrt(l2);
                const double l  = l2 * rl;
                const double f_mag = exvfam_derivative(g, l, sigma, radius);
                if(f_mag == 0.0) {continue;}
                const double c = f_mag * rl;
                for(int k=0; k<3; ++k)
                {
                    const double f = rij[k] * c;
                    force[3*i+k] += f;
                    force[3*j+k] -= f;
                }
                energy += exvfam_potential(g, l, sigma, radius);
            }
            else
            {
                energy += exvfam_potential(g, sqrt(l2), sigma, radius);
            }
        }
    }
    return energy;
}

/* The Lennard-Jones family through the generic pair loop
 * (GlobalPairInteraction.hpp:148-213): WCAPotential (WCAPotential.hpp:37-58),
 * LennardJonesAttractivePotential (LennardJonesAttractivePotential.hpp:36-70),
 * UniformLennardJonesPotential (UniformLennardJonesPotential.hpp:41-61; one
 * sigma and epsilon for every pair, kept here as equal per-particle values). */
static const double ORC_SIXTH_ROOT_OF_TWO = 1.12246204831;

static double ljfam_derivative(int kind, double r, double sigma, double epsilon, double cutoff_ratio)
{
    if(kind == ORC_WCA)
    {
        if(sigma * ORC_SIXTH_ROOT_OF_TWO < r) {return 0;}
        const double rinv = 1 / r;
        const double r1s1 = sigma * rinv;
        const double r3s3 = r1s1 * r1s1 * r1s1;
        const double r6s6 = r3s3 * r3s3;
        return 24 * epsilon * (r6s6 * (1 - 2 * r6s6)) * rinv;
    }
    if(kind == ORC_LJ_ATTRACTIVE)
    {
        if(r < sigma * ORC_SIXTH_ROOT_OF_TWO || sigma * cutoff_ratio < r) {return 0;}
        const double rinv = 1 / r;
        const double sr1 = sigma * rinv;
        const double sr3 = sr1 * sr1 * sr1;
        const double sr6 = sr3 * sr3;
        return 24 * epsilon * (sr6 - 2 * sr6 * sr6) * rinv;
    }
    /* ORC_LJ_UNIFORM */
    if(sigma * cutoff_ratio < r) {return 0;}
    const double rinv = 1 / r;
    const double sr1  = sigma * rinv;
    const double sr3  = sr1 * sr1 * sr1;
    const double sr6  = sr3 * sr3;
    return (epsilon * 24) * sr6 * (1 - 2 * sr6) * rinv;
}

static double ljfam_potential(int kind, double r, double sigma, double epsilon, double cutoff_ratio,
                              double coef_at_cutoff)
{
    if(kind == ORC_WCA)
    {
        if(sigma * ORC_SIXTH_ROOT_OF_TWO < r) {return 0;}
        const double r1s1 = sigma / r;
        const double r3s3 = r1s1 * r1s1 * r1s1;
        const double r6s6 = r3s3 * r3s3;
        return 4 * epsilon * (r6s6 * (r6s6 - 1) + 0.25);
    }
    if(kind == ORC_LJ_ATTRACTIVE)
    {
        if(r < sigma * ORC_SIXTH_ROOT_OF_TWO) {return -epsilon;}
        if(sigma * cutoff_ratio < r) {return 0;}
        const double sr1 = sigma / r;
        const double sr3 = sr1 * sr1 * sr1;
        const double sr6 = sr3 * sr3;
        return 4 * epsilon * (sr6 * (sr6 - 1) - coef_at_cutoff);
    }
    if(sigma * cutoff_ratio < r) {return 0;}
    const double sr1 = sigma / r;
    const double sr3 = sr1 * sr1 * sr1;
    const double sr6 = sr3 * sr3;
    return (epsilon * 4) * (sr6 * (sr6 - 1) - coef_at_cutoff);
}

static double ljfam_force(const orc_state* st, const orc_global* g, const double* pos,
                          double* force, int need_force)
{
    double energy = 0;
    for(int64_t q=0; q+1<g->np; ++q)
    {
        const int64_t i = g->idx[q];
        for(int64_t m=g->lb[i]; m<g->le[i]; ++m)
        {
            const int64_t j = g->nbr[m];
            const double sigma = (g->pp0[i] + g->pp0[j]) / 2;       /* LorentzBerthelotRule */
            const double e1 = g->pp1[i], e2 = g->pp1[j];
            const double epsilon = (e1 == e2) ? e1 : sqrt(e1 * e2);
            double rij[3];
            adjust_direction(st, pos + 3*i, pos + 3*j, rij);
            const double l2 = length_sq(rij);
            if(need_force)
            {
                const double rl = 1.0 / sqrt(l2);
                const double l  = l2 * rl;
                const double f_mag = ljfam_derivative(g->kind, l, sigma, epsilon, g->cutoff_ratio);
                if(f_mag == 0.0) {continue;}
                const double c = f_mag * rl;
                for(int k=0; k<3; ++k)
                {
                    const double f = rij[k] * c;
                    force[3*i+k] += f;
                    force[3*j+k] -= f;
                }
                energy += ljfam_potential(g->kind, l, sigma, epsilon, g->cutoff_ratio, g->coef_at_cutoff);
            }
            else
            {
                energy += ljfam_potential(g->kind, sqrt(l2), sigma, epsilon, g->cutoff_ratio,
                                          g->coef_at_cutoff);
            }
        }
    }
    return energy;
}

/* forcefield/global/GlobalPairLennardJonesInteraction.hpp:148-198 with the
 * Lorentz-Berthelot rule of ParameterList.hpp:240-251 */
static double lj_force(const orc_state* st, const orc_global* g, const double* pos,
                       double* force, int need_force)
{
    if(g->kind != ORC_LJ) {return ljfam_force(st, g, pos, force, need_force);}
    const double coef_at_cutoff  = g->coef_at_cutoff;
    const double cutoff_ratio    = g->cutoff_ratio;
    const double cutoff_ratio_sq = cutoff_ratio * cutoff_ratio;
    double energy = 0;
    for(int64_t q=0; q+1<g->np; ++q)
    {
        const int64_t i = g->idx[q];
        for(int64_t m=g->lb[i]; m<g->le[i]; ++m)
        {
            const int64_t j = g->nbr[m];
            const double sigma = (g->pp0[i] + g->pp0[j]) / 2;
            const double e1 = g->pp1[i], e2 = g->pp1[j];
            const double epsilon = (e1 == e2) ? e1 : sqrt(e1 * e2);
            double rij[3];
            adjust_direction(st, pos + 3*i, pos + 3*j, rij);
            const double l_sq = length_sq(rij);
            const double sigma_sq = sigma * sigma;
            if(sigma_sq * cutoff_ratio_sq < l_sq) {continue;}
            if(need_force)
            {
                const double rcp_l_sq = 1 / l_sq;
                const double s2l2 = sigma_sq * rcp_l_sq;
                const double s6l6 = s2l2 * s2l2 * s2l2;
                const double coef = 24 * epsilon * (s6l6 - 2 * s6l6 * s6l6) * rcp_l_sq;
                for(int k=0; k<3; ++k)
                {
                    const double f = rij[k] * coef;
                    force[3*i+k] += f;
                    force[3*j+k] -= f;
                }
                energy += 4 * epsilon * (s6l6 * s6l6 - s6l6 - coef_at_cutoff);
            }
            else
            {
                const double s2l2 = sigma_sq / l_sq;
                const double s6l6 = s2l2 * s2l2 * s2l2;
                energy += 4 * epsilon * (s6l6 * s6l6 - s6l6 - coef_at_cutoff);
            }
        }
    }
    return energy;
}

/* forcefield/local/BondLengthInteraction.hpp:178-199 with HarmonicPotential */
static double bond_force(const orc_state* st, const double* pos, double* force, int need_force)
{
    double energy = 0;
    for(int64_t b=0; b<st->nbond; ++b)
    {
        const int64_t i0 = st->bond_idx[2*b], i1 = st->bond_idx[2*b+1];
        const double k = st->bond_k[b], v0 = st->bond_v0[b];
        double dpos[3];
        adjust_direction(st, pos + 3*i0, pos + 3*i1, dpos);
        const double len2 = length_sq(dpos);
        if(!need_force)    /* calc_energy :114-124 */
        {
            const double dv = sqrt(len2) - v0;
            energy += k * dv * dv;
            continue;
        }
        const double rlen = 1.0 / sqrt(len2);
        const double len  = len2 * rlen;
        const double frc  = -1 * (2 * k * (len - v0));
        const double dv   = len - v0;
        energy += k * dv * dv;
        const double c = frc * rlen;
        for(int d=0; d<3; ++d)
        {
            const double f = dpos[d] * c;
            force[3*i0+d] -= f;
            force[3*i1+d] += f;
        }
    }
    return energy;
}

static inline double clampd(double x, double lo, double hi)
{
    /* math/functions.hpp:18-22: std::min(std::max(x, low), high) */
    const double a = (x < lo) ? lo : x;
    return (hi < a) ? hi : a;
}

/* forcefield/local/BondAngleInteraction.hpp:129-188 with HarmonicPotential */
static double angle_force(const orc_state* st, const double* pos, double* force, int need_force)
{
    const double abs_tol = 1e-8;     /* math/constants.hpp:26 */
    double energy = 0;
    for(int64_t a=0; a<st->nangle; ++a)
    {
        const int64_t i0 = st->angle_idx[3*a], i1 = st->angle_idx[3*a+1], i2 = st->angle_idx[3*a+2];
        const double k = st->angle_k[a], v0 = st->angle_v0[a];
        const double* p0 = pos + 3*i0; const double* p1 = pos + 3*i1; const double* p2 = pos + 3*i2;
        double r_ij[3], r_kj[3];
        adjust_direction(st, p1, p0, r_ij);
        adjust_direction(st, p1, p2, r_kj);
        if(!need_force)   /* calc_energy :190-214 */
        {
            const double lsq_rji = length_sq(r_ij);
            const double lsq_rjk = length_sq(r_kj);
            const double dot = r_ij[0] * r_kj[0] + r_ij[1] * r_kj[1] + r_ij[2] * r_kj[2];
            const double dot_reg = dot * (1.0 / sqrt(lsq_rji * lsq_rjk));
            const double th = acos(clampd(dot_reg, -1, 1));
            energy += k * (th - v0) * (th - v0);
            continue;
        }
        const double inv_ij = 1.0 / sqrt(length_sq(r_ij));
        const double inv_kj = 1.0 / sqrt(length_sq(r_kj));
        double rij_reg[3], rkj_reg[3];
        for(int d=0; d<3; ++d) {rij_reg[d] = r_ij[d] * inv_ij; rkj_reg[d] = r_kj[d] * inv_kj;}
        const double dot_ijk = rij_reg[0] * rkj_reg[0] + rij_reg[1] * rkj_reg[1] + rij_reg[2] * rkj_reg[2];
        const double cos_theta = clampd(dot_ijk, -1, 1);
        const double theta = acos(cos_theta);
        const double coef  = -(2 * k * (theta - v0));
        const double dv = theta - v0;
        energy += k * dv * dv;
        const double sin_theta = sin(theta);
        const double coef_inv_sin = coef / (sin_theta < abs_tol ? abs_tol : sin_theta);
        double Fi[3], Fk[3];
        const double ci = coef_inv_sin * inv_ij, ck = coef_inv_sin * inv_kj;
        for(int d=0; d<3; ++d)
        {
            Fi[d] = ci * (cos_theta * rij_reg[d] - rkj_reg[d]);
            Fk[d] = ck * (cos_theta * rkj_reg[d] - rij_reg[d]);
        }
        for(int d=0; d<3; ++d)
        {
            const double Fj = -Fi[d] - Fk[d];
            force[3*i0+d] += Fi[d];
            force[3*i1+d] += Fj;
            force[3*i2+d] += Fk[d];
        }
    }
    return energy;
}

static inline void cross(const double* a, const double* b, double* c)
{
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}
static inline double dot3(const double* a, const double* b)
{
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

/* forcefield/local/DihedralAngleInteraction.hpp:157-227 with CosinePotential
 * (forcefield/local/CosinePotential.hpp:29-39) */
static double dihd_force(const orc_state* st, const double* pos, double* force, int need_force)
{
    double energy = 0;
    for(int64_t a=0; a<st->ndihd; ++a)
    {
        const int64_t i0 = st->dihd_idx[4*a], i1 = st->dihd_idx[4*a+1];
        const int64_t i2 = st->dihd_idx[4*a+2], i3 = st->dihd_idx[4*a+3];
        const double K = st->dihd_k[a], v0 = st->dihd_v0[a];
        const int32_t nn = st->dihd_n[a];
        const double* r_i = pos + 3*i0; const double* r_j = pos + 3*i1;
        const double* r_k = pos + 3*i2; const double* r_l = pos + 3*i3;
        double r_ij[3], r_kj[3], r_lk[3], r_kl[3];
        adjust_direction(st, r_j, r_i, r_ij);
        adjust_direction(st, r_j, r_k, r_kj);
        adjust_direction(st, r_k, r_l, r_lk);
        for(int d=0; d<3; ++d) {r_kl[d] = -1.0 * r_lk[d];}
        if(!need_force)   /* calc_energy :129-155 */
        {
            const double r_kj_lensq_inv = 1.0 / length_sq(r_kj);
            double nvec[3];
            cross(r_kj, r_kl, nvec);
            double R[3], S[3];
            const double c1 = dot3(r_ij, r_kj) * r_kj_lensq_inv;
            const double c2 = dot3(r_lk, r_kj) * r_kj_lensq_inv;
            for(int d=0; d<3; ++d) {R[d] = r_ij[d] - c1 * r_kj[d]; S[d] = r_lk[d] - c2 * r_kj[d];}
            const double dot_RS = dot3(R, S) * (1.0 / sqrt(length_sq(R) * length_sq(S)));
            const double cos_phi = clampd(dot_RS, -1.0, 1.0);
            const double phi = copysign(acos(cos_phi), dot3(r_ij, nvec));
            energy += K * (1 + cos(nn * (phi - v0)));
            continue;
        }
        const double r_kj_lensq  = length_sq(r_kj);
        const double r_kj_rlen   = 1.0 / sqrt(r_kj_lensq);
        const double r_kj_rlensq = r_kj_rlen * r_kj_rlen;
        const double r_kj_len    = r_kj_rlen * r_kj_lensq;
        double m[3], nv[3];
        cross(r_ij, r_kj, m);
        cross(r_kj, r_kl, nv);
        const double m_lensq = length_sq(m);
        const double n_lensq = length_sq(nv);
        const double dot_mn  = dot3(m, nv) * (1.0 / sqrt(m_lensq * n_lensq));
        const double cos_phi = clampd(dot_mn, -1, 1);
        const double phi     = copysign(acos(cos_phi), dot3(r_ij, nv));
        const double dv      = phi - v0;
        const double coef    = -(-K * nn * sin(nn * dv));
        energy += K * (1 + cos(nn * dv));
        const double cfi = coef * r_kj_len / m_lensq;
        const double cfl = -coef * r_kj_len / n_lensq;
        double Fi[3], Fl[3];
        for(int d=0; d<3; ++d) {Fi[d] = cfi * m[d]; Fl[d] = cfl * nv[d];}
        const double coef_ijk = dot3(r_ij, r_kj) * r_kj_rlensq;
        const double coef_jkl = dot3(r_kl, r_kj) * r_kj_rlensq;
        for(int d=0; d<3; ++d)
        {
            const double Fj = (coef_ijk - 1.0) * Fi[d] - coef_jkl * Fl[d];
            const double Fk = (coef_jkl - 1.0) * Fl[d] - coef_ijk * Fi[d];
            force[3*i0+d] += Fi[d];
            force[3*i1+d] += Fj;
            force[3*i2+d] += Fk;
            force[3*i3+d] += Fl[d];
        }
    }
    return energy;
}

static double eval_term(const orc_state* st, int term, const double* pos, double* force, int need_force)
{
    switch(term)
    {
        case ORC_TERM_BOND:     return bond_force (st, pos, force, need_force);
        case ORC_TERM_ANGLE:    return angle_force(st, pos, force, need_force);
        case ORC_TERM_DIHEDRAL: return dihd_force (st, pos, force, need_force);
        case ORC_TERM_EXV: return st->g[0].on ? exv_force(st, &st->g[0], pos, force, need_force) : 0;
        case ORC_TERM_DH:  return st->g[1].on ? dh_force (st, &st->g[1], pos, force, need_force) : 0;
        case ORC_TERM_LJ:  return st->g[2].on ? lj_force (st, &st->g[2], pos, force, need_force) : 0;
        default: return 0;
    }
}

static int term_on(const orc_state* st, int term)
{
    switch(term)
    {
        case ORC_TERM_BOND:     return st->nbond  > 0;
        case ORC_TERM_ANGLE:    return st->nangle > 0;
        case ORC_TERM_DIHEDRAL: return st->ndihd  > 0;
        default: return term >= ORC_TERM_EXV && term <= ORC_TERM_LJ && st->g[term - ORC_TERM_EXV].on;
    }
}

/* Forces of one term on `pos` with a list built on `pos` (the reference builds
 * its lists in ForceField::initialize on the same coordinates). */
int orc_term_force(const orc_state* st_, int term, const double* pos, double* force, double* energy)
{
    orc_state* st = (orc_state*)st_;
    if(!term_on(st, term)) {return -1;}
    memset(force, 0, sizeof(double) * 3 * st->n);
    if(term >= ORC_TERM_EXV)
    {
        orc_global* g = &st->g[term - ORC_TERM_EXV];
        /* build a list on pos without disturbing the dynamics' list */
        int64_t* lb = calloc((size_t)st->n, sizeof(int64_t));
        int64_t* le = calloc((size_t)st->n, sizeof(int64_t));
        int64_t* nbr = NULL; int64_t c = 0;
        half_list(st, term - ORC_TERM_EXV, pos, lb, le, &nbr, &c);
        orc_global tmp = *g;
        tmp.lb = lb; tmp.le = le; tmp.nbr = nbr;
        *energy = term == ORC_TERM_EXV ? exv_force(st, &tmp, pos, force, 1) :
                  term == ORC_TERM_DH  ? dh_force (st, &tmp, pos, force, 1) :
                                         lj_force (st, &tmp, pos, force, 1);
        free(lb); free(le); free(nbr);
        return 0;
    }
    *energy = eval_term(st, term, pos, force, 1);
    return 0;
}

int orc_term_energy(const orc_state* st_, int term, const double* pos, double* energy)
{
    orc_state* st = (orc_state*)st_;
    if(!term_on(st, term)) {return -1;}
    if(term >= ORC_TERM_EXV)
    {
        orc_global* g = &st->g[term - ORC_TERM_EXV];
        int64_t* lb = calloc((size_t)st->n, sizeof(int64_t));
        int64_t* le = calloc((size_t)st->n, sizeof(int64_t));
        int64_t* nbr = NULL; int64_t c = 0;
        half_list(st, term - ORC_TERM_EXV, pos, lb, le, &nbr, &c);
        orc_global tmp = *g;
        tmp.lb = lb; tmp.le = le; tmp.nbr = nbr;
        *energy = term == ORC_TERM_EXV ? exv_force(st, &tmp, pos, NULL, 0) :
                  term == ORC_TERM_DH  ? dh_force (st, &tmp, pos, NULL, 0) :
                                         lj_force (st, &tmp, pos, NULL, 0);
        free(lb); free(le); free(nbr);
        return 0;
    }
    *energy = eval_term(st, term, pos, NULL, 0);
    return 0;
}

/* ForceField::calc_force order: local (bond, angle, dihedral) then global
 * (EXV, DH, LJ) on the current lists (core/ForceField.hpp:101-109). */
static void calc_force(orc_state* st)
{
    for(int t=0; t<ORC_NTERMS; ++t)
    {
        if(term_on(st, t)) {eval_term(st, t, st->pos, st->force, 1);}
    }
}

/* ---------------------------------------------------------------- philox */

void orc_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for(int r=0; r<10; ++r)
    {
        if(r) {k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;}
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

void orc_gaussian3(uint64_t seed, uint64_t particle, uint64_t step, double out[3])
{
    const uint32_t ctr[4] = {(uint32_t)particle, (uint32_t)(particle >> 32),
                             (uint32_t)step,     (uint32_t)(step >> 32)};
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t x[4];
    orc_philox4x32(ctr, key, x);
    const double two32 = 2.3283064365386963e-10;   /* 2^-32 */
    const double u0 = ((double)x[0] + 0.5) * two32;
    const double u1 = (double)x[1] * two32;
    const double u2 = ((double)x[2] + 0.5) * two32;
    const double u3 = (double)x[3] * two32;
    const double pi = 3.14159265358979323846;
    const double r0 = sqrt(-2.0 * log(u0));
    const double r1 = sqrt(-2.0 * log(u2));
    out[0] = r0 * cos(pi * (2.0 * u1));
    out[1] = r0 * sin(pi * (2.0 * u1));
    out[2] = r1 * cos(pi * (2.0 * u3));
}

/* ------------------------------------------------------------ integrator */

/* Noise coefficients of the Langevin integrators.
 * BAOAB: BAOABLangevinIntegrator::reset_parameters (:73-99),
 *   exp(-gamma dt) and sqrt(kB T (1 - exp(-2 gamma dt)) / m).
 * UnderdampedLangevin: UnderdampedLangevinIntegrator::update (:281-300), the
 *   acceleration noise sigma = sqrt(2 kB T / dt) sqrt(gamma / m), kept in
 *   noise_coeff (exp_gamma_dt unused).
 * G-JF: GJFNVTLangevinIntegrator::reset_parameters (:111-136), with alpha in
 *   gamma: b = 1 / (1 + alpha dt / 2m) in gjf_b, beta = sqrt(2 alpha kB T dt)
 *   in noise_coeff, a = 1 - alpha b dt / m in exp_gamma_dt. */
static void noise_parameters(orc_state* st)
{
    const double kBT = st->kB * st->T;
    const double ul_coef = sqrt(2 * st->kB * st->T / st->dt);
    for(int64_t i=0; i<st->n; ++i)
    {
        if(st->s.integrator == ORC_UNDERDAMPED)
        {
            st->exp_gamma_dt[i] = 1.0;
            st->noise_coeff[i]  = ul_coef * sqrt(st->gamma[i] * st->rmass[i]);
            continue;
        }
        if(st->s.integrator == ORC_GJF)
        {
            const double alpha = st->gamma[i], m = st->mass[i];
            st->gjf_b[i]        = 1.0 / (1.0 + alpha * st->dt * 0.5 / m);
            st->noise_coeff[i]  = sqrt(2 * alpha * kBT * st->dt);
            st->exp_gamma_dt[i] = 1.0 - alpha * st->gjf_b[i] * st->dt / m;
            continue;
        }
        const double gamma_dt = -1 * st->gamma[i] * st->dt;
        st->exp_gamma_dt[i] = exp(gamma_dt);
        st->noise_coeff[i]  = sqrt(kBT * (1 - exp(2 * gamma_dt)) * st->rmass[i]);
    }
}

/* a = f/m + sigma R (UnderdampedLangevinIntegrator::initialize, :160-181, and
 * the closing of step, :252-264), with the Philox noise of counter `ctr` */
static void underdamped_accel(orc_state* st, int64_t i, uint64_t ctr)
{
    double R[3];
    orc_gaussian3(st->s.seed, (uint64_t)i, ctr, R);
    for(int d=0; d<3; ++d)
    {
        st->accel[3*i+d] = st->force[3*i+d] * st->rmass[i] + R[d] * st->noise_coeff[i];
    }
}

/* BAOABLangevinIntegrator::initialize (:135-168); VelocityVerletIntegrator and
 * UnderdampedLangevinIntegrator::initialize (:160-181) have the same force
 * evaluation, the latter followed by the first acceleration (noise counter 0). */
int orc_init_dynamics(orc_state* st)
{
    noise_parameters(st);
    memset(st->force, 0, sizeof(double) * 3 * st->n);
    calc_force(st);
    st->step = 0;
    if(st->s.integrator == ORC_UNDERDAMPED)
    {
        for(int64_t i=0; i<st->n; ++i) {underdamped_accel(st, i, st->step);}
    }
    return 0;
}

/* BAOABLangevinIntegrator::update (:47-58) after the system's temperature
 * attribute changed (SimulatedAnnealingSimulator::step,
 * core/SimulatedAnnealingSimulator.hpp:144-154): reset_parameters with the new
 * temperature.  The DebyeHuckel parameters keep the old temperature, as in the
 * reference. */
void orc_set_temperature(orc_state* st, double T)
{
    st->T = T;
    noise_parameters(st);
}

/* GlobalPairInteraction::reduce_margin -> ...GridCellList::reduce_margin */
static void reduce_margin(orc_state* st, double dmargin)
{
    for(int gi=0; gi<3; ++gi)
    {
        orc_global* g = &st->g[gi];
        if(!g->on) {continue;}
        g->current_margin -= dmargin;
        if(g->current_margin < 0) {make_list(st, gi);}
    }
}

int orc_run(orc_state* st, int64_t nsteps)
{
    const int64_t n = st->n;
    const double halfdt = st->halfdt;
    for(int64_t s=0; s<nsteps; ++s)
    {
        double largest_disp2 = 0.0;
        if(st->s.integrator == ORC_VV)   /* VelocityVerletIntegrator.hpp:90-135 */
        {
            for(int64_t i=0; i<n; ++i)
            {
                double disp[3];
                const double c = halfdt * st->rmass[i];
                for(int d=0; d<3; ++d)
                {
                    st->vel[3*i+d] += c * st->force[3*i+d];
                    disp[d] = st->dt * st->vel[3*i+d];
                    st->pos[3*i+d] = st->pos[3*i+d] + disp[d];
                    st->force[3*i+d] = 0;
                }
                adjust_position(st, st->pos + 3*i);
                const double d2 = length_sq(disp);
                largest_disp2 = largest_disp2 < d2 ? d2 : largest_disp2;
            }
        }
        else if(st->s.integrator == ORC_UNDERDAMPED)   /* UnderdampedLangevinIntegrator.hpp:198-221 */
        {
            const double dt = st->dt, halfdt2 = dt * dt / 2;
            for(int64_t i=0; i<n; ++i)
            {
                const double gdo2 = st->gamma[i] * halfdt;
                const double omg  = 1 - gdo2;
                const double* a = st->accel + 3*i;
                double disp[3];
                for(int d=0; d<3; ++d)
                {
                    disp[d] = (dt * omg) * st->vel[3*i+d] + halfdt2 * a[d];
                    st->pos[3*i+d] = st->pos[3*i+d] + disp[d];
                    st->vel[3*i+d] *= omg * (omg * omg + gdo2);
                    st->vel[3*i+d] += (halfdt * omg) * a[d];
                    st->force[3*i+d] = 0;
                }
                adjust_position(st, st->pos + 3*i);
                const double d2 = length_sq(disp);
                largest_disp2 = largest_disp2 < d2 ? d2 : largest_disp2;
            }
        }
        else if(st->s.integrator == ORC_GJF)   /* GJFNVTLangevinIntegrator.hpp:175-204 */
        {
            const double dt = st->dt;
            for(int64_t i=0; i<n; ++i)
            {
                const double rm = st->rmass[i], r2m = 0.5 * rm;
                const double b = st->gjf_b[i], a = st->exp_gamma_dt[i];
                double R[3], beta[3], dp[3];
                orc_gaussian3(st->s.seed, (uint64_t)i, st->step, R);
                for(int d=0; d<3; ++d) {beta[d] = R[d] * st->noise_coeff[i];}
                for(int d=0; d<3; ++d)
                {
                    double* v = st->vel + 3*i+d;
                    const double f = st->force[3*i+d];
                    dp[d] = (b * dt) * (*v + r2m * (dt * f + beta[d]));
                    st->pos[3*i+d] = st->pos[3*i+d] + dp[d];
                    *v = a * (*v + (dt * r2m) * f) + b * rm * beta[d];
                    st->force[3*i+d] = 0;
                }
                adjust_position(st, st->pos + 3*i);
                const double d2 = length_sq(dp);
                largest_disp2 = largest_disp2 < d2 ? d2 : largest_disp2;
            }
        }
        else if(st->s.integrator == ORC_GBAOAB)   /* gBAOABLangevinIntegrator.hpp:318-420, no constraints */
        {
            for(int64_t i=0; i<n; ++i)
            {
                double R[3], dp[3];
                orc_gaussian3(st->s.seed, (uint64_t)i, st->step, R);
                const double rm = st->rmass[i];
                double* p = st->pos + 3*i;
                double* v = st->vel + 3*i;
                for(int d=0; d<3; ++d) {v[d] += halfdt * rm * st->force[3*i+d];}            /* B */
                double q[3];
                for(int d=0; d<3; ++d) {q[d] = p[d] + halfdt * v[d];}                        /* A */
                for(int d=0; d<3; ++d) {v[d] *= st->exp_gamma_dt[i];}                        /* O */
                for(int d=0; d<3; ++d) {v[d] += st->noise_coeff[i] * R[d];}
                for(int d=0; d<3; ++d) {q[d] = q[d] + halfdt * v[d];}                        /* A */
                for(int d=0; d<3; ++d)
                {
                    dp[d] = q[d] - p[d];              /* position(i) - old_position_[i] */
                    p[d] = q[d];
                    st->force[3*i+d] = 0;
                }
                adjust_position(st, p);
                const double d2 = length_sq(dp);
                largest_disp2 = largest_disp2 < d2 ? d2 : largest_disp2;
            }
        }
        else                              /* BAOABLangevinIntegrator.hpp:170-240 */
        {
            for(int64_t i=0; i<n; ++i)
            {
                double R[3];
                orc_gaussian3(st->s.seed, (uint64_t)i, st->step, R);
                const double rm = st->rmass[i];
                const double expgt = st->exp_gamma_dt[i];
                const double noise = st->noise_coeff[i];
                double dp[3];
                for(int d=0; d<3; ++d)
                {
                    double v = st->vel[3*i+d];
                    v += halfdt * rm * st->force[3*i+d];
                    dp[d] = 0.0 + halfdt * v;
                    v *= expgt;
                    v += noise * R[d];
                    dp[d] += halfdt * v;
                    st->vel[3*i+d] = v;
                    st->pos[3*i+d] = st->pos[3*i+d] + dp[d];
                    st->force[3*i+d] = 0;
                }
                adjust_position(st, st->pos + 3*i);
                const double d2 = length_sq(dp);
                largest_disp2 = largest_disp2 < d2 ? d2 : largest_disp2;
            }
        }
        reduce_margin(st, 2 * sqrt(largest_disp2));
        calc_force(st);
        if(st->s.integrator == ORC_UNDERDAMPED)   /* UnderdampedLangevinIntegrator.hpp:252-264 */
        {
            for(int64_t i=0; i<n; ++i)
            {
                underdamped_accel(st, i, st->step + 1);
                const double k = halfdt * (1 - st->gamma[i] * halfdt);
                for(int d=0; d<3; ++d) {st->vel[3*i+d] += k * st->accel[3*i+d];}
            }
        }
        else    /* BAOAB, velocity Verlet; G-JF's (dt 0.5 / m) f (:211-218) is the same product */
        {
            for(int64_t i=0; i<n; ++i)
            {
                const double c = halfdt * st->rmass[i];
                for(int d=0; d<3; ++d) {st->vel[3*i+d] += c * st->force[3*i+d];}
            }
        }
        st->step++;
    }
    return 0;
}

void orc_get_state(const orc_state* st, double* pos, double* vel, double* force)
{
    if(pos)   {memcpy(pos,   st->pos,   sizeof(double) * 3 * st->n);}
    if(vel)   {memcpy(vel,   st->vel,   sizeof(double) * 3 * st->n);}
    if(force) {memcpy(force, st->force, sizeof(double) * 3 * st->n);}
}

int64_t orc_rebuild_count(const orc_state* st, int term)
{
    const int gi = term - ORC_TERM_EXV;
    if(gi < 0 || gi > 2 || !st->g[gi].on) {return -1;}
    return st->g[gi].rebuilds;
}
