/*
 * Test infrastructure (oracle): plain-C restatement of the LPM-CPP implicit quasi-static step.
 * This file is the checker for the device path (tests, smoke check and the CPU-baseline leg
 * of the benchmark only).  It is single-threaded and evaluates every expression in the
 * reference's operator order; built with -ffp-contract=off it reproduces the reference's
 * arithmetic bit for bit, which tests/test_oracle_golden.py pins against the reference's own
 * build (oracle/_ref) through the committed fixtures in tests/golden/.
 *
 * Citations are paths inside the LPM-CPP tree.  MKL calls are replaced by the semantics the
 * oracle/shim stand-in implements (in-order sums; RCI CG test on squared norms).
 */
#include "lpm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define EPS 1e-6 /* include/lpm.h:41 */

struct lpmo_problem
{
    int n, dim, lattice, ptype, nsv, nlayer;
    double radius, cutoff[2], pvol;
    int nneighbors;
    double el[9];
    /* particles */
    double *xyz, *xyz0, *xyz_last, *pin, *pex, *stress;
    double *damage, *damage_last, *damage_visual, *ddot_local, *ddot_nonlocal, *sv, *sv_last;
    int *cons, *type, *nb, *nb0;
    int *bstart;
    double *dLe_total, *TdLe_total, *cs_sum; /* n*2, n*2, n*2*3 */
    /* bonds, owner-major: layer-0 list then layer-1 list, each in ascending p2 */
    long nbonds;
    int *bp2, *blayer, *brev;
    double *dis0, *dis, *dis_last, *dL, *dLe, *dLp, *dLp_last, *bstrain, *Kn, *Tv, *cs, *bforce, *bforce_last,
        *bdamage, *bdamage_last;
    /* connections */
    int *cstart, *conns, *nlq;
    /* nonlocal neighbours */
    int *nlstart, *nlist;
    /* material */
    double E, mu, critical_bstrain, sigmay, xi, H, A, damage_threshold, nonlocal_L;
    double k0, k1; /* ParticleElasticDamage damage surface (particle_elastic_damage.h:27) */
    double fA, fB, fd; /* ParticleFatigueHCF rate law (particle_fatigue_hcf.h:19) */
    int undamaged_type, max_iter, tangent;
    double tol, cg_rtol, cg_atol;
    long long cg_maxit;
    /* stiffness, reference layout (stiffness.h:24-26) */
    long long *K_pointer, *IK, *JK;
    double *K, *residual;
    double reaction_sq; /* in-order sum of squares of the whole reaction history (solver.h:25,64) */
};

/* ---------------------------------------------------------------- unit cell (unit_cell.h:27-122) */
static void set_cell(lpmo_problem *p, int lattice, double r)
{
    p->lattice = lattice;
    p->radius = r;
    double s2 = sqrt(2.0), s3 = sqrt(3.0);
    switch (lattice)
    {
    case LPMO_SQUARE2D: /* unit_cell.h:44-58 */
    {
        double e[9] = {1. / 2., -1. / 2., 0., 0., 0., 1. / 2., 0., 1. / 12., -1. / 12.};
        memcpy(p->el, e, sizeof e);
        p->dim = 2;
        p->nneighbors = 8;
        p->cutoff[0] = 2.0 * r;
        p->cutoff[1] = 2.0 * s2 * r;
        p->pvol = 4 * pow(r, 2);
        break;
    }
    case LPMO_HEXAGON2D: /* unit_cell.h:60-74 */
    {
        double e[9] = {s3 / 12.0, -s3 / 12.0, 0., -s3 / 144.0, s3 / 48.0, 0.0, 0.0, 0.0, 1.0};
        memcpy(p->el, e, sizeof e);
        p->dim = 2;
        p->nneighbors = 12;
        p->cutoff[0] = 2.0 * r;
        p->cutoff[1] = 2.0 * s3 * r;
        p->pvol = 2 * s3 * pow(r, 2);
        break;
    }
    case LPMO_SC3D: /* unit_cell.h:76-90 */
    {
        double e[9] = {1, -1, -1.0, 0.0, 0.0, 1., 0.0, 1 / 18.0, -1 / 18.0};
        memcpy(p->el, e, sizeof e);
        p->dim = 3;
        p->nneighbors = 18;
        p->cutoff[0] = 2.0 * r;
        p->cutoff[1] = 2.0 * s2 * r;
        p->pvol = pow(2 * r, 3);
        break;
    }
    case LPMO_FCC3D: /* unit_cell.h:92-106 */
    {
        double e[9] = {0.0, 0.0, s2, s2 / 4, -s2 / 4, -s2 / 4, 0.0, s2 / 24, -s2 / 24};
        memcpy(p->el, e, sizeof e);
        p->dim = 3;
        p->nneighbors = 18;
        p->cutoff[0] = 2.0 * r;
        p->cutoff[1] = 2.0 * s2 * r;
        p->pvol = 4.0 * s2 * pow(r, 3);
        break;
    }
    default: /* BCC, unit_cell.h:108-122 */
    {
        double e[9] = {0.0, 0.0, s3, 1 / s3, -1 / s3, 0., 0.0, s3 / 14, s3 / 14};
        memcpy(p->el, e, sizeof e);
        p->dim = 3;
        p->nneighbors = 14;
        p->cutoff[0] = 2.0 * r;
        p->cutoff[1] = 4.0 / s3 * r;
        p->pvol = 32.0 * s3 / 9.0 * pow(r, 3);
        break;
    }
    }
}

/* ------------------------------------------------------------- generators (utilities.h:15-310) */
void lpmo_rmatrix(int f, const double a[3], double R[9])
{
    double a1 = a[0], a2 = a[1], a3 = a[2];
    if (f == 0) /* utilities.h:36-52 */
    {
        R[0] = cos(a2) * cos(a3);
        R[1] = -cos(a2) * sin(a3);
        R[2] = sin(a2);
        R[3] = cos(a1) * sin(a3) + sin(a1) * sin(a2) * cos(a3);
        R[4] = cos(a1) * cos(a3) - sin(a1) * sin(a2) * sin(a3);
        R[5] = -sin(a1) * cos(a2);
        R[6] = sin(a1) * sin(a3) - cos(a1) * sin(a2) * cos(a3);
        R[7] = sin(a1) * cos(a3) + cos(a1) * sin(a2) * sin(a3);
        R[8] = cos(a1) * cos(a2);
    }
    else if (f == 1) /* utilities.h:53-69 */
    {
        R[0] = -cos(a1) * cos(a2) * cos(a3) - sin(a1) * sin(a3);
        R[1] = cos(a3) * sin(a1) - sin(a3) * cos(a2) * cos(a1);
        R[2] = sin(a2) * cos(a1);
        R[3] = sin(a3) * cos(a1) - cos(a3) * cos(a2) * sin(a1);
        R[4] = -cos(a1) * cos(a3) - sin(a1) * cos(a2) * sin(a3);
        R[5] = sin(a2) * sin(a1);
        R[6] = cos(a3) * sin(a2);
        R[7] = sin(a3) * sin(a2);
        R[8] = cos(a2);
    }
    else /* Bunge, utilities.h:70-88 */
    {
        R[0] = -sin(a1) * cos(a2) * sin(a3) + cos(a1) * cos(a3);
        R[1] = -sin(a3) * cos(a1) - cos(a3) * cos(a2) * sin(a1);
        R[2] = sin(a1) * sin(a2);
        R[3] = cos(a3) * sin(a1) + sin(a3) * cos(a2) * cos(a1);
        R[4] = -sin(a1) * sin(a3) + cos(a1) * cos(a2) * cos(a3);
        R[5] = -cos(a1) * sin(a2);
        R[6] = sin(a2) * sin(a3);
        R[7] = sin(a2) * cos(a3);
        R[8] = cos(a2);
    }
}

/* y = R p with the oracle's dgemv semantics (alpha = 1, beta = 0, in-order sums) */
static void rot(const double R[9], const double p[3], double y[3])
{
    for (int i = 0; i < 3; ++i)
    {
        double s = 0.0;
        for (int j = 0; j < 3; ++j)
            s += R[3 * i + j] * p[j];
        y[i] = 1.0 * s;
    }
}

static long push(double *out, long cap, long n, double x, double y, double z)
{
    if (out && n < cap)
    {
        out[3 * n] = x;
        out[3 * n + 1] = y;
        out[3 * n + 2] = z;
    }
    return n + 1;
}

long lpmo_generate(int lattice, double radius, const double box[6], const double R[9], double *out, long cap)
{
    long n = 0;
    double p[3] = {0, 0, 0}, q[3];
    if (lattice == LPMO_SQUARE2D) /* utilities.h:93-125 */
    {
        double a = sqrt(pow(box[1] - box[0], 2) + pow(box[3] - box[2], 2));
        double bt[6] = {-a, a, -a, a, -a, a};
        double hx = 2 * radius, hy = hx;
        int first = (int)floor((bt[1] - bt[0]) / hx);
        int rows = (int)floor((bt[3] - bt[2]) / hy);
        for (int j = 1; j <= rows; j++)
        {
            p[1] = bt[2] + hy * (j - 1) + radius;
            for (int i = 1; i <= first; i++)
            {
                p[0] = bt[0] + hx * (i - 1) + radius;
                rot(R, p, q);
                if (q[0] >= box[0] && q[0] <= box[1] && q[1] >= box[2] && q[1] <= box[3])
                    n = push(out, cap, n, q[0], q[1], 0);
            }
        }
        return n;
    }
    if (lattice == LPMO_HEXAGON2D) /* utilities.h:127-177 */
    {
        double a = sqrt(pow(box[1] - box[0], 2) + pow(box[3] - box[2], 2));
        double bt[6] = {-a, a, -a, a, -a, a};
        double hx = 2 * radius, hy = hx * sqrt(3.0) / 2.0;
        int first = 1 + (int)floor((bt[1] - bt[0]) / hx);
        int rows = 1 + (int)floor((bt[3] - bt[2]) / hy);
        for (int j = 1; j <= rows; j++)
        {
            double y = bt[2] + hy * (j - 1);
            int cnt = (j % 2 == 1) ? first : first - 1;
            for (int i = 1; i <= cnt; i++)
            {
                double x = (j % 2 == 1) ? bt[0] + hx * (i - 1) : bt[0] + hx * (2 * i - 1) / 2.0;
                double pp[3] = {x, y, 0};
                rot(R, pp, q);
                if (q[0] >= box[0] && q[0] <= box[1] && q[1] >= box[2] && q[1] <= box[3])
                    n = push(out, cap, n, q[0], q[1], q[2]);
            }
        }
        return n;
    }
    if (lattice == LPMO_SC3D) /* utilities.h:179-220; x starts at box[0], y and z at -a */
    {
        double a = sqrt(pow(box[1] - box[0], 2) + pow(box[3] - box[2], 2) + pow(box[5] - box[4], 2));
        double bt[6] = {-a, a, -a, a, -a, a};
        double hx = 2 * radius, hy = hx, hz = hx;
        int first = 1 + (int)floor((bt[1] - bt[0]) / hx);
        int rows = 1 + (int)floor((bt[3] - bt[2]) / hy);
        int layers = 1 + (int)floor((bt[5] - bt[4]) / hz);
        for (int k = 1; k <= layers; k++)
        {
            p[2] = bt[4] + hz * (k - 1);
            for (int j = 1; j <= rows; j++)
            {
                p[1] = bt[2] + hy * (j - 1);
                for (int i = 1; i <= first; i++)
                {
                    p[0] = box[0] + hx * (i - 1);
                    rot(R, p, q);
                    if (q[0] >= box[0] && q[0] <= box[1] && q[1] >= box[2] && q[1] <= box[3] && q[2] >= box[4] &&
                        q[2] <= box[5])
                        n = push(out, cap, n, q[0], q[1], q[2]);
                }
            }
        }
        return n;
    }
    if (lattice == LPMO_FCC3D) /* utilities.h:222-310 */
    {
        double a = sqrt(pow(box[1] - box[0], 2) + pow(box[3] - box[2], 2) + pow(box[5] - box[4], 2));
        double bt[6] = {-a, a, -a, a, -a, a};
        double hx = 4 * radius / sqrt(2.0), hy = hx, hz = hx;
        int first = 1 + (int)floor((bt[1] - bt[0]) / hx);
        int rows = 1 + (int)floor((bt[3] - bt[2]) / (hy / 2.0));
        int layers = 1 + (int)floor((bt[5] - bt[4]) / (hz / 2.0));
        for (int k = 1; k <= layers; k++)
        {
            double z = bt[4] + hz / 2.0 * (k - 1);
            for (int j = 1; j <= rows; j++)
            {
                double y = bt[2] + hy / 2.0 * (j - 1);
                int full = ((k % 2 == 1) == (j % 2 == 1));
                int cnt = full ? first : first - 1;
                for (int i = 1; i <= cnt; i++)
                {
                    double x = full ? bt[0] + hx * (i - 1) : bt[0] + hx * (i - 1) + hx / 2.0;
                    double pp[3] = {x, y, z};
                    rot(R, pp, q);
                    if (q[0] >= box[0] && q[0] <= box[1] && q[1] >= box[2] && q[1] <= box[3] && q[2] >= box[4] &&
                        q[2] <= box[5])
                        n = push(out, cap, n, q[0], q[1], q[2]);
                }
            }
        }
        return n;
    }
    /* BCC: the reference has no C++ generator.  Cubic cell a = 4r/sqrt(3) (nearest-neighbour
     * distance 2r, unit_cell.h:108-122), corner sites then body-centre sites per z layer of
     * half cells, laid out like the FCC generator: on [-d, d]^3, rotated, clipped to the box. */
    {
        double a = sqrt(pow(box[1] - box[0], 2) + pow(box[3] - box[2], 2) + pow(box[5] - box[4], 2));
        double bt[6] = {-a, a, -a, a, -a, a};
        double h = 4 * radius / sqrt(3.0);
        int first = 1 + (int)floor((bt[1] - bt[0]) / h);
        int layers = 1 + (int)floor((bt[5] - bt[4]) / (h / 2.0));
        for (int k = 1; k <= layers; k++)
        {
            double z = bt[4] + h / 2.0 * (k - 1);
            int corner = (k % 2 == 1);
            int cnt = corner ? first : first - 1;
            for (int j = 1; j <= cnt; j++)
            {
                double y = corner ? bt[2] + h * (j - 1) : bt[2] + h * (j - 1) + h / 2.0;
                for (int i = 1; i <= cnt; i++)
                {
                    double x = corner ? bt[0] + h * (i - 1) : bt[0] + h * (i - 1) + h / 2.0;
                    double pp[3] = {x, y, z};
                    rot(R, pp, q);
                    if (q[0] >= box[0] && q[0] <= box[1] && q[1] >= box[2] && q[1] <= box[3] && q[2] >= box[4] &&
                        q[2] <= box[5])
                        n = push(out, cap, n, q[0], q[1], q[2]);
                }
            }
        }
        return n;
    }
}

/* particle.h:277-280 */
static double dist(const double *a, const double *b)
{
    return sqrt(pow((a[0] - b[0]), 2) + pow((a[1] - b[1]), 2) + pow((a[2] - b[2]), 2));
}

/* ------------------------------------------------------------- construction */
typedef struct
{
    int id, layer;
    double d;
} cand_t;

static int cmp_cand(const void *a, const void *b)
{
    const cand_t *x = (const cand_t *)a, *y = (const cand_t *)b;
    return (x->id > y->id) - (x->id < y->id);
}

static int cmp_int(const void *a, const void *b)
{
    int x = *(const int *)a, y = *(const int *)b;
    return (x > y) - (x < y);
}

/* Assembly::createBonds (assembly.h:213-234): all pairs, bond if d < 1.01*cutoff[1] and i != j,
 * layer 0 if d < 1.01*cutoff[0]; per particle the lists follow ascending partner id.  The
 * candidates come from a uniform cell grid (cells no smaller than the cutoff), then sorted by
 * id, which yields exactly the lists of the all-pairs loop. */
static int build_bonds(lpmo_problem *p)
{
    const int n = p->n;
    const double rc1 = 1.01 * p->cutoff[1], rc0 = 1.01 * p->cutoff[0];
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k)
        {
            lo[k] = fmin(lo[k], p->xyz0[3 * i + k]);
            hi[k] = fmax(hi[k], p->xyz0[3 * i + k]);
        }
    double h = rc1 * 1.0001;
    int nc[3];
    long ncell = 1;
    for (int k = 0; k < 3; ++k)
    {
        nc[k] = (int)floor((hi[k] - lo[k]) / h) + 1;
        if (nc[k] < 1)
            nc[k] = 1;
        ncell *= nc[k];
    }
    int *cell_of = (int *)malloc(sizeof(int) * n);
    int *cstart = (int *)calloc(ncell + 1, sizeof(int));
    int *clist = (int *)malloc(sizeof(int) * n);
    for (int i = 0; i < n; ++i)
    {
        int c[3];
        for (int k = 0; k < 3; ++k)
        {
            c[k] = (int)floor((p->xyz0[3 * i + k] - lo[k]) / h);
            if (c[k] >= nc[k])
                c[k] = nc[k] - 1;
            if (c[k] < 0)
                c[k] = 0;
        }
        cell_of[i] = (c[2] * nc[1] + c[1]) * nc[0] + c[0];
        cstart[cell_of[i] + 1]++;
    }
    for (long c = 0; c < ncell; ++c)
        cstart[c + 1] += cstart[c];
    int *fill = (int *)malloc(sizeof(int) * ncell);
    memcpy(fill, cstart, sizeof(int) * ncell);
    for (int i = 0; i < n; ++i)
        clist[fill[cell_of[i]]++] = i;
    free(fill);

    int cap = 64;
    cand_t *cand = (cand_t *)malloc(sizeof(cand_t) * cap);
    long btotal = 0, bcap = (long)n * 20 + 16;
    int *bp2 = (int *)malloc(sizeof(int) * bcap), *bl = (int *)malloc(sizeof(int) * bcap);
    double *bd = (double *)malloc(sizeof(double) * bcap);
    p->bstart = (int *)malloc(sizeof(int) * (n + 1));
    p->nb = (int *)malloc(sizeof(int) * n);
    p->nb0 = (int *)malloc(sizeof(int) * n);
    for (int i = 0; i < n; ++i)
    {
        int ci = cell_of[i];
        int cx = ci % nc[0], cy = (ci / nc[0]) % nc[1], cz = ci / (nc[0] * nc[1]);
        int nf = 0;
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx)
                {
                    int x = cx + dx, y = cy + dy, z = cz + dz;
                    if (x < 0 || y < 0 || z < 0 || x >= nc[0] || y >= nc[1] || z >= nc[2])
                        continue;
                    long c = ((long)z * nc[1] + y) * nc[0] + x;
                    for (int q = cstart[c]; q < cstart[c + 1]; ++q)
                    {
                        int j = clist[q];
                        double d = dist(p->xyz0 + 3 * i, p->xyz0 + 3 * j);
                        if ((d < rc1) && (i != j))
                        {
                            if (nf == cap)
                            {
                                cap *= 2;
                                cand = (cand_t *)realloc(cand, sizeof(cand_t) * cap);
                            }
                            cand[nf].id = j;
                            cand[nf].layer = (d < rc0) ? 0 : 1;
                            cand[nf].d = d;
                            nf++;
                        }
                    }
                }
        qsort(cand, nf, sizeof(cand_t), cmp_cand);
        if (btotal + nf > bcap)
        {
            bcap = 2 * (btotal + nf);
            bp2 = (int *)realloc(bp2, sizeof(int) * bcap);
            bl = (int *)realloc(bl, sizeof(int) * bcap);
            bd = (double *)realloc(bd, sizeof(double) * bcap);
        }
        p->bstart[i] = (int)btotal;
        int c0 = 0;
        for (int L = 0; L < 2; ++L)
            for (int q = 0; q < nf; ++q)
                if (cand[q].layer == L)
                {
                    bp2[btotal] = cand[q].id;
                    bl[btotal] = L;
                    bd[btotal] = cand[q].d;
                    btotal++;
                    if (L == 0)
                        c0++;
                }
        p->nb[i] = nf;
        p->nb0[i] = c0;
    }
    p->bstart[n] = (int)btotal;
    p->nbonds = btotal;
    p->bp2 = bp2;
    p->blayer = bl;
    p->dis0 = bd;
    free(cand);
    free(cell_of);
    free(cstart);
    free(clist);
    return 0;
}

/* Assembly::readBond (assembly.h:391-424): the caller's lists in their own order, each bond
 * with dis = Particle::distanceTo (particle.h) and the layer it is listed under */
static void build_bonds_user(lpmo_problem *p, const lpmo_desc *d)
{
    const int n = p->n;
    long tot = 0;
    for (int i = 0; i < n; ++i)
        tot += d->bond_nb0[i] + d->bond_nb1[i];
    p->bstart = (int *)malloc(sizeof(int) * (n + 1));
    p->nb = (int *)malloc(sizeof(int) * n);
    p->nb0 = (int *)malloc(sizeof(int) * n);
    p->bp2 = (int *)malloc(sizeof(int) * (tot + 1));
    p->blayer = (int *)malloc(sizeof(int) * (tot + 1));
    p->dis0 = (double *)malloc(sizeof(double) * (tot + 1));
    long b = 0;
    for (int i = 0; i < n; ++i)
    {
        p->bstart[i] = (int)b;
        p->nb0[i] = d->bond_nb0[i];
        p->nb[i] = d->bond_nb0[i] + d->bond_nb1[i];
        for (int q = 0; q < p->nb[i]; ++q, ++b)
        {
            const int j = d->bond_p2[b];
            p->bp2[b] = j;
            p->blayer[b] = (q < d->bond_nb0[i]) ? 0 : 1;
            p->dis0[b] = dist(p->xyz0 + 3 * i, p->xyz0 + 3 * j);
        }
    }
    p->bstart[n] = (int)b;
    p->nbonds = b;
}

#define B0(p, i) ((p)->bstart[i])
#define B1(p, i) ((p)->bstart[i] + (p)->nb0[i])
#define BE(p, i) ((p)->bstart[(i) + 1])
#define LB(p, i, L) ((L) == 0 ? B0(p, i) : B1(p, i))
#define LE(p, i, L) ((L) == 0 ? B1(p, i) : BE(p, i))

/* Assembly::updateConnections (assembly.h:237-266) */
static void build_conns(lpmo_problem *p)
{
    const int n = p->n;
    p->cstart = (int *)malloc(sizeof(int) * (n + 1));
    p->nlq = (int *)malloc(sizeof(int) * n);
    long cap = (long)n * 32 + 16, tot = 0;
    int *cl = (int *)malloc(sizeof(int) * cap);
    int tcap = 256;
    int *tmp = (int *)malloc(sizeof(int) * tcap);
    for (int i = 0; i < n; ++i)
    {
        int m = 0;
        for (int L = 0; L < 2; ++L)
            for (int b = LB(p, i, L); b < LE(p, i, L); ++b)
            {
                int k = p->bp2[b];
                int need = m + 1 + (LE(p, k, L) - LB(p, k, L));
                if (need > tcap)
                {
                    tcap = 2 * need;
                    tmp = (int *)realloc(tmp, sizeof(int) * tcap);
                }
                tmp[m++] = k;
                for (int c = LB(p, k, L); c < LE(p, k, L); ++c)
                    tmp[m++] = p->bp2[c];
            }
        qsort(tmp, m, sizeof(int), cmp_int);
        int u = 0;
        for (int q = 0; q < m; ++q)
            if (u == 0 || tmp[q] != tmp[u - 1])
                tmp[u++] = tmp[q];
        if (tot + u > cap)
        {
            cap = 2 * (tot + u);
            cl = (int *)realloc(cl, sizeof(int) * cap);
        }
        p->cstart[i] = (int)tot;
        int self = -1;
        for (int q = 0; q < u; ++q)
        {
            cl[tot + q] = tmp[q];
            if (tmp[q] == i)
                self = q;
        }
        p->nlq[i] = (self < 0) ? 0 : u - self;
        tot += u;
    }
    p->cstart[n] = (int)tot;
    p->conns = cl;
    free(tmp);
}

/* opposite bond: first bond of p2's same-layer list pointing back (particle.h:207-209) */
static void build_rev(lpmo_problem *p)
{
    p->brev = (int *)malloc(sizeof(int) * (p->nbonds + 1));
    for (int i = 0; i < p->n; ++i)
        for (int L = 0; L < 2; ++L)
            for (int b = LB(p, i, L); b < LE(p, i, L); ++b)
            {
                int j = p->bp2[b];
                p->brev[b] = -1;
                for (int c = LB(p, j, L); c < LE(p, j, L); ++c)
                    if (p->bp2[c] == i)
                    {
                        p->brev[b] = c;
                        break;
                    }
            }
}

/* Assembly::searchNonlocalNeighbors (assembly.h:118-130), all pairs in id order */
static void build_nonlocal(lpmo_problem *p, double ratio)
{
    const int n = p->n;
    p->nlstart = (int *)malloc(sizeof(int) * (n + 1));
    long cap = 1024, tot = 0;
    int *l = (int *)malloc(sizeof(int) * cap);
    for (int i = 0; i < n; ++i)
    {
        p->nlstart[i] = (int)tot;
        if (ratio > 0)
            for (int j = 0; j < n; ++j)
                if (dist(p->xyz + 3 * i, p->xyz + 3 * j) < ratio * p->nonlocal_L)
                {
                    if (tot == cap)
                    {
                        cap *= 2;
                        l = (int *)realloc(l, sizeof(int) * cap);
                    }
                    l[tot++] = j;
                }
    }
    p->nlstart[n] = (int)tot;
    p->nlist = l;
}

#define ALLOCD(x, cnt) ((x) = (double *)calloc((size_t)(cnt) + 1, sizeof(double)))

lpmo_problem *lpmo_create(const lpmo_desc *d)
{
    lpmo_problem *p = (lpmo_problem *)calloc(1, sizeof(lpmo_problem));
    const int n = d->n;
    p->n = n;
    p->nlayer = 2;
    p->ptype = d->ptype;
    set_cell(p, d->lattice, d->radius);
    /* J2: 7 (particle_j2plasticity.h); fatigue HCF: [0] largest energy so far, [1] / [2] the
     * smallest / largest energy of the current cycle (particle_fatigue_hcf.h:16) */
    p->nsv = (d->ptype == LPMO_J2) ? 7 : (d->ptype == LPMO_FATIGUE_HCF) ? 3 : 1;
    ALLOCD(p->xyz, 3 * n);
    ALLOCD(p->xyz0, 3 * n);
    ALLOCD(p->xyz_last, 3 * n);
    ALLOCD(p->pin, 3 * n);
    ALLOCD(p->pex, 3 * n);
    ALLOCD(p->stress, 6 * n);
    ALLOCD(p->damage, n);
    ALLOCD(p->damage_last, n);
    ALLOCD(p->damage_visual, n);
    ALLOCD(p->ddot_local, n);
    ALLOCD(p->ddot_nonlocal, n);
    ALLOCD(p->sv, p->nsv * n);
    ALLOCD(p->sv_last, p->nsv * n);
    ALLOCD(p->dLe_total, 2 * n);
    ALLOCD(p->TdLe_total, 2 * n);
    ALLOCD(p->cs_sum, 6 * n);
    p->cons = (int *)calloc(3 * (size_t)n + 1, sizeof(int));
    p->type = (int *)calloc((size_t)n + 1, sizeof(int));
    memcpy(p->xyz, d->xyz, sizeof(double) * 3 * n);
    memcpy(p->xyz0, d->xyz, sizeof(double) * 3 * n);
    memcpy(p->xyz_last, d->xyz, sizeof(double) * 3 * n);
    if (d->type)
        memcpy(p->type, d->type, sizeof(int) * n);
    if (d->ptype == LPMO_FATIGUE_HCF)
        for (int i = 0; i < n; ++i) /* state_var = state_var_last = {0, INT_MAX, 0} (particle_fatigue_hcf.h:27-28) */
        {
            p->sv[3 * i + 1] = 2147483647.0;
            p->sv_last[3 * i + 1] = 2147483647.0;
        }

    if (d->bond_nb0 && d->bond_nb1 && d->bond_p2)
        build_bonds_user(p, d);
    else
        build_bonds(p);
    build_conns(p);
    build_rev(p);
    const long nb = p->nbonds;
    ALLOCD(p->dis, nb);
    ALLOCD(p->dis_last, nb);
    ALLOCD(p->dL, nb);
    ALLOCD(p->dLe, nb);
    ALLOCD(p->dLp, nb);
    ALLOCD(p->dLp_last, nb);
    ALLOCD(p->bstrain, nb);
    ALLOCD(p->Kn, nb);
    ALLOCD(p->Tv, nb);
    ALLOCD(p->cs, 3 * nb);
    ALLOCD(p->bforce, nb);
    ALLOCD(p->bforce_last, nb);
    ALLOCD(p->bdamage, nb);
    ALLOCD(p->bdamage_last, nb);
    /* Bond(p1, p2, layer, dis) (bond.h:59-72) */
    for (int i = 0; i < n; ++i)
        for (int b = B0(p, i); b < BE(p, i); ++b)
        {
            int j = p->bp2[b];
            p->dis[b] = p->dis0[b];
            p->dis_last[b] = p->dis0[b];
            for (int k = 0; k < 3; ++k)
                p->cs[3 * b + k] = (p->xyz[3 * i + k] - p->xyz[3 * j + k]) / p->dis0[b];
        }

    /* material: setParticleProperty (particle_elastic.h:70-108, particle_j2plasticity.h:154-198) */
    p->E = d->E;
    p->mu = d->mu;
    p->critical_bstrain = d->critical_bstrain;
    p->sigmay = d->sigmay;
    p->xi = d->xi;
    p->H = d->H;
    p->A = d->A;
    /* never assigned for J2 in the reference (particle_j2plasticity.h:22); ParticleElasticDamage
     * takes it from setParticleProperty (particle_elastic_damage.h:186) */
    p->damage_threshold =
        (d->ptype == LPMO_ELASTIC_DAMAGE || d->ptype == LPMO_FATIGUE_HCF) ? d->damage_threshold : 0;
    p->fA = d->fatigue_A;
    p->fB = d->fatigue_B;
    p->fd = d->fatigue_d;
    p->k0 = d->k0;
    p->k1 = d->k1;
    p->nonlocal_L = d->nonlocal_L;
    double E = d->E, mu = d->mu, Ce[3], KnTv[3];
    if (d->C11 > 0 && d->ptype != LPMO_J2)
    {
        Ce[0] = d->C11;
        Ce[1] = d->C12;
        Ce[2] = d->C44;
    }
    else if (!d->plane_stress)
    {
        Ce[0] = E * (1.0 - mu) / (1.0 + mu) / (1.0 - 2.0 * mu);
        Ce[1] = E * mu / (1.0 + mu) / (1.0 - 2.0 * mu);
        Ce[2] = E / 2.0 / (1.0 + mu);
    }
    else
    {
        Ce[0] = E / (1.0 - mu) / (1.0 + mu);
        Ce[1] = E * mu / (1.0 + mu) / (1.0 - mu);
        Ce[2] = E / 2.0 / (1.0 + mu);
    }
    double alpha = (p->dim == 2) ? 1.0 : p->radius;
    for (int r = 0; r < 3; ++r)
    {
        double s = 0.0;
        for (int c = 0; c < 3; ++c)
            s += p->el[3 * r + c] * Ce[c];
        KnTv[r] = alpha * s;
    }
    for (long b = 0; b < nb; ++b)
    {
        if (p->lattice == LPMO_HEXAGON2D)
        {
            p->Kn[b] = KnTv[0];
            p->Tv[b] = KnTv[1];
        }
        else
        {
            p->Kn[b] = KnTv[p->blayer[b]];
            p->Tv[b] = KnTv[2];
        }
    }
    p->undamaged_type = d->undamaged_type;
    p->max_iter = d->max_iter;
    p->tangent = d->tangent;
    p->tol = d->tol_iter;
    p->cg_rtol = d->cg_rtol;
    p->cg_atol = d->cg_atol;
    p->cg_maxit = d->cg_maxit;
    build_nonlocal(p, d->nonlocal_cutoff_ratio);

    /* Stiffness::initialize (stiffness.h:55-71) */
    const int dim = p->dim;
    p->K_pointer = (long long *)calloc((size_t)n + 1, sizeof(long long));
    p->K_pointer[0] = 0;
    for (int i = 0; i < n; ++i)
        p->K_pointer[i + 1] = p->K_pointer[i] + (long long)dim * dim * p->nlq[i] - (dim == 2 ? 1 : 3);
    p->IK = (long long *)calloc((size_t)dim * n + 1, sizeof(long long));
    p->JK = (long long *)calloc((size_t)p->K_pointer[n] + 1, sizeof(long long));
    ALLOCD(p->K, p->K_pointer[n]);
    ALLOCD(p->residual, dim * n);
    return p;
}

void lpmo_destroy(lpmo_problem *p)
{
    if (!p)
        return;
    void *ptrs[] = {p->xyz, p->xyz0, p->xyz_last, p->pin, p->pex, p->stress, p->damage, p->damage_last,
                    p->damage_visual, p->ddot_local, p->ddot_nonlocal, p->sv, p->sv_last, p->cons, p->type, p->nb,
                    p->nb0, p->bstart, p->dLe_total, p->TdLe_total, p->cs_sum, p->bp2, p->blayer, p->brev,
                    p->dis0, p->dis, p->dis_last, p->dL, p->dLe, p->dLp, p->dLp_last, p->bstrain, p->Kn, p->Tv,
                    p->cs, p->bforce, p->bforce_last, p->bdamage, p->bdamage_last, p->cstart, p->conns, p->nlq,
                    p->nlstart, p->nlist, p->K_pointer, p->IK, p->JK, p->K, p->residual};
    for (size_t k = 0; k < sizeof ptrs / sizeof ptrs[0]; ++k)
        free(ptrs[k]);
    free(p);
}

int lpmo_dim(const lpmo_problem *p) { return p->dim; }
long lpmo_nbonds(const lpmo_problem *p) { return p->nbonds; }
long lpmo_nconn_total(const lpmo_problem *p) { return p->cstart[p->n]; }
long long lpmo_nnz_upper(const lpmo_problem *p) { return p->K_pointer[p->n]; }
int lpmo_nstate_var(const lpmo_problem *p) { return p->nsv; }

void lpmo_get_bonds(const lpmo_problem *p, int *nb0, int *nb1, int *p2)
{
    for (int i = 0; i < p->n; ++i)
    {
        nb0[i] = p->nb0[i];
        nb1[i] = p->nb[i] - p->nb0[i];
    }
    memcpy(p2, p->bp2, sizeof(int) * p->nbonds);
}

void lpmo_get_conns(const lpmo_problem *p, int *nconn, int *nlq, int *conns)
{
    for (int i = 0; i < p->n; ++i)
    {
        nconn[i] = p->cstart[i + 1] - p->cstart[i];
        nlq[i] = p->nlq[i];
    }
    memcpy(conns, p->conns, sizeof(int) * p->cstart[p->n]);
}

/* ------------------------------------------------------------- per-iteration physics */
/* Particle::updateBondsGeometry (particle.h:164-181) -> Bond::updatebGeometry (bond.h:30-39) */
void lpmo_update_geometry(lpmo_problem *p)
{
    for (int i = 0; i < p->n; ++i)
        for (int L = 0; L < 2; ++L)
        {
            double s = 0, ts = 0, cx = 0, cy = 0, cz = 0;
            for (int b = LB(p, i, L); b < LE(p, i, L); ++b)
            {
                int j = p->bp2[b];
                const double *x1 = p->xyz + 3 * i, *x2 = p->xyz + 3 * j;
                int broken = fabs(p->bdamage[b] - 1.0) < EPS;
                double dis = dist(x1, x2);
                p->dis[b] = dis;
                p->dL[b] = broken ? 0.0 : (dis - p->dis0[b]);
                p->bstrain[b] = broken ? 0.0 : (p->dL[b] / dis);
                p->dLe[b] = broken ? 0.0 : (dis - p->dis0[b] - p->dLp[b]);
                p->cs[3 * b] = broken ? 0.0 : ((x1[0] - x2[0]) / dis);
                p->cs[3 * b + 1] = broken ? 0.0 : ((x1[1] - x2[1]) / dis);
                p->cs[3 * b + 2] = broken ? 0.0 : ((x1[2] - x2[2]) / dis);
                s += p->dLe[b];
                ts += p->Tv[b] * p->dLe[b];
                cx += p->cs[3 * b];
                cy += p->cs[3 * b + 1];
                cz += p->cs[3 * b + 2];
            }
            p->dLe_total[2 * i + L] = s;
            p->TdLe_total[2 * i + L] = ts;
            p->cs_sum[6 * i + 3 * L] = cx;
            p->cs_sum[6 * i + 3 * L + 1] = cy;
            p->cs_sum[6 * i + 3 * L + 2] = cz;
        }
}

static double std_max(double a, double b) { return (a < b) ? b : a; }

/* Assembly::updateForceState (assembly.h:179-191) */
void lpmo_update_force_state(lpmo_problem *p)
{
    const int n = p->n;
    /* ParticleElastic::updateBondsForce (particle_elastic.h:38-50);
     * ParticleJ2Plasticity::updateBondsForce (particle_j2plasticity.h:63-76) and
     * ParticleElasticDamage::updateBondsForce (particle_elastic_damage.h:80-91) and
     * ParticleFatigueHCF::updateBondsForce (particle_fatigue_hcf.h:66-80): bond damage is the
     * largest of its own and its two particles' */
    for (int i = 0; i < n; ++i)
        for (int b = B0(p, i); b < BE(p, i); ++b)
        {
            int L = p->blayer[b];
            double f = 2. * p->Kn[b] * p->dLe[b] + 2. * p->Tv[b] * p->dLe_total[2 * i + L];
            if (p->ptype == LPMO_J2 || p->ptype == LPMO_ELASTIC_DAMAGE || p->ptype == LPMO_FATIGUE_HCF)
                p->bdamage[b] = std_max(p->bdamage[b], std_max(p->damage[i], p->damage[p->bp2[b]]));
            f *= (1.0 - p->bdamage[b]);
            p->bforce[b] = f;
        }
    for (int i = 0; i < n; ++i)
    {
        /* Particle::updateParticleForce (particle.h:198-215) */
        double P[3] = {0., 0., 0.};
        for (int b = B0(p, i); b < BE(p, i); ++b)
        {
            double fo = p->bforce[p->brev[b]];
            P[0] += p->cs[3 * b] * 0.5 * (p->bforce[b] + fo);
            P[1] += p->cs[3 * b + 1] * 0.5 * (p->bforce[b] + fo);
            P[2] += p->cs[3 * b + 2] * 0.5 * (p->bforce[b] + fo);
        }
        for (int k = 0; k < 3; ++k)
            p->pin[3 * i + k] = P[k];
        /* Particle::updateParticleStress (particle.h:218-240) */
        double S[6] = {0, 0, 0, 0, 0, 0};
        double V_m = p->pvol * p->nb[i] / p->nneighbors;
        for (int b = B0(p, i); b < BE(p, i); ++b)
        {
            double fo = p->bforce[p->brev[b]];
            double cx = p->cs[3 * b], cy = p->cs[3 * b + 1], cz = p->cs[3 * b + 2], ds = p->dis[b];
            S[0] += 0.5 / V_m * (ds) * 0.5 * (p->bforce[b] + fo) * (cx) * (cx);
            S[1] += 0.5 / V_m * (ds) * 0.5 * (p->bforce[b] + fo) * (cy) * (cy);
            S[2] += 0.5 / V_m * (ds) * 0.5 * (p->bforce[b] + fo) * (cz) * (cz);
            S[3] += 0.5 / V_m * (ds) * 0.5 * (p->bforce[b] + fo) * (cy) * (cz);
            S[4] += 0.5 / V_m * (ds) * 0.5 * (p->bforce[b] + fo) * (cx) * (cz);
            S[5] += 0.5 / V_m * (ds) * 0.5 * (p->bforce[b] + fo) * (cx) * (cy);
        }
        for (int k = 0; k < 6; ++k)
            p->stress[6 * i + k] = S[k];
        /* Particle::updateParticleDamageVisual (particle.h:151-161) */
        double dv = 0;
        for (int b = B0(p, i); b < BE(p, i); ++b)
            dv += p->bdamage[b];
        p->damage_visual[i] = dv / (double)p->nb[i];
    }
}

/* ParticleJ2Plasticity::updateParticleStateVariables (particle_j2plasticity.h:78-140);
 * Particle::updateParticleStateVariables is a no-op for elastic particles (particle.h:62) */
void lpmo_update_state_var(lpmo_problem *p)
{
    if (p->ptype == LPMO_FATIGUE_HCF)
    {
        /* ParticleFatigueHCF::updateParticleStateVariables (particle_fatigue_hcf.h:128-145) with
         * calcEqEnergy (:83-125), which returns the total energy: the spring energy of each bond
         * plus the volumetric term of each layer, per modified volume (its split into
         * dilatational and distortional parts does not reach the result) */
        for (int i = 0; i < p->n; ++i)
        {
            const double V_m = p->pvol * p->nb[i] / p->nneighbors;
            double energy = 0;
            for (int L = 0; L < 2; ++L)
            {
                const int lo = L == 0 ? B0(p, i) : B0(p, i) + p->nb0[i], hi = L == 0 ? B0(p, i) + p->nb0[i] : BE(p, i);
                for (int b = lo; b < hi; ++b)
                    energy += 0.5 * (p->Kn[b] * p->dLe[b] * p->dLe[b]) / V_m;
                energy += 0.5 * p->TdLe_total[2 * i + L] * p->dLe_total[2 * i + L] / V_m;
            }
            double *sv = p->sv + 3 * i;
            sv[1] = (sv[1] < energy) ? sv[1] : energy; /* std::min(curr, sv[1]) */
            sv[2] = (energy < sv[2]) ? sv[2] : energy; /* std::max(curr, sv[2]) */
            sv[0] = (sv[2] < sv[0]) ? sv[0] : sv[2];   /* std::max(sv[2], sv[0]) */
            if (sv[2] - sv[1] > 0)
                p->ddot_local[i] = p->fA * pow(sv[0], p->fB) * pow(sv[2] - sv[1], p->fd);
            else
                p->ddot_local[i] = 0;
        }
        return;
    }
    if (p->ptype == LPMO_ELASTIC_DAMAGE)
    {
        /* ParticleElasticDamage::updateParticleStateVariables (particle_elastic_damage.h:159-170)
         * with calcStrainEnergyDensity (:93-108): state_var[0] = strain energy density, the
         * local damage rate from its increase past the damage surface */
        for (int i = 0; i < p->n; ++i)
        {
            const double V_m = p->pvol * p->nb[i] / p->nneighbors;
            double energy = 0;
            for (int L = 0; L < 2; ++L)
            {
                const int lo = L == 0 ? B0(p, i) : B0(p, i) + p->nb0[i], hi = L == 0 ? B0(p, i) + p->nb0[i] : BE(p, i);
                for (int b = lo; b < hi; ++b)
                    energy += 0.5 * (p->Kn[b] * p->dLe[b] * p->dLe[b]) / V_m;
                energy += 0.5 * p->TdLe_total[2 * i + L] * p->dLe_total[2 * i + L] / V_m;
            }
            p->sv[i] = energy;
            const double delta = p->sv[i] - p->sv_last[i];
            const double f = p->sv[i] - p->k1 * p->damage[i] - p->k0;
            p->ddot_local[i] = (f > 0 && delta > 0) ? (1 / p->k1) * delta : 0;
        }
        return;
    }
    if (p->ptype != LPMO_J2)
        return;
    for (int i = 0; i < p->n; ++i)
    {
        double *sv = p->sv + 7 * i;
        double st[6], dpl[6] = {0, 0, 0, 0, 0, 0};
        double sigma_m, sigma_eq = 0.0, triax = 0.0, dlambda = 0.0;
        for (int j = 0; j < 6; ++j)
            st[j] = p->stress[6 * i + j];
        sigma_m = 1.0 / 3.0 * (st[0] + st[1] + st[2]);
        for (int j = 0; j < 3; j++)
            st[j] -= sigma_m;
        for (int j = 0; j < 6; j++)
            st[j] -= sv[j + 1];
        for (int j = 0; j < 6; j++)
        {
            if (j < 3)
                sigma_eq += st[j] * st[j];
            else
                sigma_eq += 2.0 * st[j] * st[j];
        }
        sigma_eq = sqrt(3.0 / 2.0 * sigma_eq);
        double yield = sigma_eq - (p->sigmay + (1.0 - p->xi) * p->H * sv[0]);
        double G = p->E / 2 / (1 + p->mu);
        if (yield > 0.0)
            dlambda = yield / (3 * G + p->H);
        sv[0] += dlambda;
        for (int j = 0; j < 6; j++)
            if (fabs(sigma_eq) > EPS)
            {
                dpl[j] = dlambda * 1.5 * st[j] / sigma_eq;
                sv[j + 1] += 2. / 3. * p->xi * p->H * dpl[j];
            }
        for (int b = B0(p, i); b < BE(p, i); ++b)
        {
            double cx = p->cs[3 * b], cy = p->cs[3 * b + 1], cz = p->cs[3 * b + 2];
            double ddLp = p->dis[b] * (dpl[0] * cx * cx + dpl[1] * cy * cy + dpl[2] * cz * cz + 2 * dpl[3] * cy * cz +
                                       2 * dpl[4] * cx * cz + 2 * dpl[5] * cx * cy);
            p->dLp[b] += ddLp;
        }
        if (sigma_eq > EPS)
            triax = sigma_m / sigma_eq;
        p->ddot_local[i] = dlambda * (1.0 + p->A * triax);
    }
}

/* Solver::updateRR (solver.h:112-126) + cblas_dnrm2 of the residual (solver.h:63,85) */
double lpmo_update_rr(lpmo_problem *p)
{
    const int dim = p->dim;
    double s = 0.0;
    for (int i = 0; i < p->n; ++i)
        for (int k = 0; k < dim; ++k)
        {
            p->residual[dim * i + k] = (1 - p->cons[3 * i + k]) * (p->pex[3 * i + k] - p->pin[3 * i + k]);
            if (p->cons[3 * i + k] == 1)
                p->reaction_sq += p->pin[3 * i + k] * p->pin[3 * i + k];
        }
    for (long q = 0; q < (long)dim * p->n; ++q)
        s += p->residual[q] * p->residual[q];
    return sqrt(s);
}

void lpmo_read_residual(const lpmo_problem *p, double *res)
{
    memcpy(res, p->residual, sizeof(double) * p->dim * p->n);
}

/* ------------------------------------------------------------- stiffness */
typedef double blk_t[3][3];

/* Particle::hasAFEMneighbor (particle.h:243-256) */
static int has_afem(const lpmo_problem *p, int i, int j, int L)
{
    for (int b1 = LB(p, i, L); b1 < LE(p, i, L); ++b1)
    {
        int k = p->bp2[b1];
        if (k == j)
            return 1;
        for (int b2 = LB(p, k, L); b2 < LE(p, k, L); ++b2)
            if (p->bp2[b2] == j)
                return 1;
    }
    return 0;
}

#define CS(b, a) (p->cs[3 * (b) + (a)])
#define SUMCS(j, L, a) (p->cs_sum[6 * (j) + 3 * (L) + (a)])

/* fdu2dxyz (derivative.h:8-45): diagonal block, upper part plus the two mirrored entries */
static void fdu2dxyz(const lpmo_problem *p, int i, blk_t K)
{
    memset(K, 0, sizeof(blk_t));
    for (int L = 0; L < 2; ++L)
        for (int b = LB(p, i, L); b < LE(p, i, L); ++b)
        {
            double D = p->bdamage[b], Kn = p->Kn[b], Tv = p->Tv[b];
            double x = CS(b, 0), y = CS(b, 1), z = CS(b, 2);
            double Sx = SUMCS(i, L, 0), Sy = SUMCS(i, L, 1), Sz = SUMCS(i, L, 2);
            K[0][0] += (1 - D) * ((Kn * x + Tv * Sx) * x + (Kn + Tv) * pow(x, 2));
            K[0][1] += (1 - D) * ((Kn * y + Tv * Sy) * x + (Kn + Tv) * y * x);
            K[0][2] += (1 - D) * ((Kn * z + Tv * Sz) * x + (Kn + Tv) * z * x);
            K[1][1] += (1 - D) * ((Kn * y + Tv * Sy) * y + (Kn + Tv) * pow(y, 2));
            K[1][2] += (1 - D) * ((Kn * z + Tv * Sz) * y + (Kn + Tv) * z * y);
            K[2][2] += (1 - D) * ((Kn * z + Tv * Sz) * z + (Kn + Tv) * pow(z, 2));
        }
    K[2][0] = K[0][2];
    K[2][1] = K[1][2];
}

/* other-bond term (derivative.h:91-99 / 188-196): bd1 gives the column cosine, bd2 the row */
static void sub_pair(const lpmo_problem *p, blk_t K, int bd1, int bd2)
{
    double t = 0.5 * ((1 - p->bdamage[bd1]) * p->Tv[bd1] + (1 - p->bdamage[bd2]) * p->Tv[bd2]);
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            K[r][c] -= t * CS(bd2, r) * CS(bd1, c);
}

/* fdu2dxyz1 / fdu2dxyz2 (derivative.h:48-142 / 145-239), layer L */
static void fdu2dxyzL(const lpmo_problem *p, int i, int j, int L, blk_t K)
{
    memset(K, 0, sizeof(blk_t));
    for (int bd1 = LB(p, i, L); bd1 < LE(p, i, L); ++bd1)
    {
        if (p->bp2[bd1] == j)
        {
            for (int bd2 = LB(p, i, L); bd2 < LE(p, i, L); ++bd2)
            {
                if (p->bp2[bd1] == p->bp2[bd2])
                {
                    double D = p->bdamage[bd2], Kn = p->Kn[bd2], Tv = p->Tv[bd2];
                    int k2 = p->bp2[bd2];
                    double x = CS(bd2, 0), y = CS(bd2, 1), z = CS(bd2, 2);
                    double Sx = SUMCS(k2, L, 0), Sy = SUMCS(k2, L, 1), Sz = SUMCS(k2, L, 2);
                    K[0][0] += (1 - D) * ((-Kn * x + Tv * Sx) * x - (Kn + Tv) * pow(x, 2));
                    K[0][1] += (1 - D) * ((-Kn * y + Tv * Sy) * x - (Kn + Tv) * y * x);
                    K[0][2] += (1 - D) * ((-Kn * z + Tv * Sz) * x - (Kn + Tv) * z * x);
                    K[1][0] += (1 - D) * ((-Kn * x + Tv * Sx) * y - (Kn + Tv) * y * x);
                    K[1][1] += (1 - D) * ((-Kn * y + Tv * Sy) * y - (Kn + Tv) * pow(y, 2));
                    K[1][2] += (1 - D) * ((-Kn * z + Tv * Sz) * y - (Kn + Tv) * z * y);
                    K[2][0] += (1 - D) * ((-Kn * x + Tv * Sx) * z - (Kn + Tv) * z * x);
                    K[2][1] += (1 - D) * ((-Kn * y + Tv * Sy) * z - (Kn + Tv) * z * y);
                    K[2][2] += (1 - D) * ((-Kn * z + Tv * Sz) * z - (Kn + Tv) * pow(z, 2));
                }
                else
                {
                    sub_pair(p, K, bd1, bd2);
                    int k = p->bp2[bd2];
                    for (int bd3 = LB(p, k, L); bd3 < LE(p, k, L); ++bd3)
                        if (p->bp2[bd3] == j)
                        {
                            /* derivative.h:105-113: row cosine from bd2, column from bd3 */
                            double t =
                                0.5 * ((1 - p->bdamage[bd3]) * p->Tv[bd3] + (1 - p->bdamage[bd2]) * p->Tv[bd2]);
                            for (int r = 0; r < 3; ++r)
                                for (int c = 0; c < 3; ++c)
                                    K[r][c] -= t * CS(bd2, r) * CS(bd3, c);
                        }
                }
            }
            return;
        }
    }
    /* derivative.h:122-139: two-hop paths i -> k -> j */
    for (int bd1 = LB(p, i, L); bd1 < LE(p, i, L); ++bd1)
    {
        int k = p->bp2[bd1];
        for (int bd2 = LB(p, k, L); bd2 < LE(p, k, L); ++bd2)
            if (p->bp2[bd2] == j)
            {
                double t = 0.5 * ((1 - p->bdamage[bd2]) * p->Tv[bd2] + (1 - p->bdamage[bd1]) * p->Tv[bd1]);
                for (int r = 0; r < 3; ++r)
                    for (int c = 0; c < 3; ++c)
                        K[r][c] -= t * CS(bd1, r) * CS(bd2, c);
            }
    }
}

/* Stiffness::localStiffnessANA (stiffness.h:109-142) */
static void local_stiffness(const lpmo_problem *p, int i, int j, blk_t K)
{
    blk_t K1, K2;
    int f1 = 0, f2 = 0;
    memset(K, 0, sizeof(blk_t));
    memset(K1, 0, sizeof(blk_t));
    memset(K2, 0, sizeof(blk_t));
    if (has_afem(p, i, j, 0))
    {
        fdu2dxyzL(p, i, j, 0, K1);
        f1 = 1;
    }
    if (has_afem(p, i, j, 1))
    {
        fdu2dxyzL(p, i, j, 1, K2);
        f2 = 1;
    }
    if (i == j)
        fdu2dxyz(p, i, K);
    else if (f1 && f2)
    {
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c)
                K[r][c] = K1[r][c] + K2[r][c];
    }
    else if (f1)
        memcpy(K, K1, sizeof(blk_t));
    else if (f2)
        memcpy(K, K2, sizeof(blk_t));
}

/* position of conn j within i's conns counted from the end (std::distance(find, end)) */
static int conn_pos(const lpmo_problem *p, int i, int j)
{
    for (int q = p->cstart[i]; q < p->cstart[i + 1]; ++q)
        if (p->conns[q] == j)
            return q - p->cstart[i];
    return -1;
}

/* Stiffness::reset + calcStiffness2D/3D (stiffness.h:74-89, 198-361), serial pi order, and
 * Stiffness::updateStiffnessDispBC (stiffness.h:364-438) when apply_bc */
void lpmo_assemble(lpmo_problem *p, int apply_bc)
{
    const int n = p->n, dim = p->dim;
    long long *Kp = p->K_pointer;
    double *Kg = p->K;
    long long *JK = p->JK;
    for (int i = 0; i < n; ++i)
        Kp[i + 1] = Kp[i] + (long long)dim * dim * p->nlq[i] - (dim == 2 ? 1 : 3);
    for (long long q = 0; q < Kp[n]; ++q)
    {
        JK[q] = 0;
        Kg[q] = 0;
    }
    for (int i = 0; i < n; ++i)
    {
        const int nlq = p->nlq[i], nconn = p->cstart[i + 1] - p->cstart[i];
        for (int idx = 0; idx < nconn; ++idx)
        {
            int j = p->conns[p->cstart[i] + idx];
            blk_t Kl;
            local_stiffness(p, i, j, Kl);
            long long base = Kp[i];
            if (dim == 3)
            {
                if (i == j)
                {
                    Kg[base] += Kl[0][0];
                    Kg[base + 1] += Kl[0][1];
                    Kg[base + 2] += Kl[0][2];
                    Kg[base + dim * nlq] += Kl[1][1];
                    Kg[base + dim * nlq + 1] += Kl[1][2];
                    Kg[base + 2 * dim * nlq - 1] += Kl[2][2];
                    JK[base] = dim * (j + 1) - 2;
                    JK[base + 1] = dim * (j + 1) - 1;
                    JK[base + 2] = dim * (j + 1);
                    JK[base + dim * nlq] = dim * (j + 1) - 1;
                    JK[base + dim * nlq + 1] = dim * (j + 1);
                    JK[base + 2 * dim * nlq - 1] = dim * (j + 1);
                }
                else if (j > i)
                {
                    int num1 = nlq - (nconn - idx);
                    long long r0 = base + dim * num1, r1 = base + dim * nlq + dim * num1 - 1,
                              r2 = base + 2 * dim * nlq + dim * num1 - 3;
                    for (int c = 0; c < 3; ++c)
                    {
                        Kg[r0 + c] += 0.5 * Kl[0][c];
                        Kg[r1 + c] += 0.5 * Kl[1][c];
                        Kg[r2 + c] += 0.5 * Kl[2][c];
                        JK[r0 + c] = dim * (j + 1) - 2 + c;
                        JK[r1 + c] = dim * (j + 1) - 2 + c;
                        JK[r2 + c] = dim * (j + 1) - 2 + c;
                    }
                }
                else
                {
                    int nlqj = p->nlq[j];
                    int num2 = nlqj - ((p->cstart[j + 1] - p->cstart[j]) - conn_pos(p, j, i));
                    long long bj = Kp[j];
                    long long r0 = bj + dim * num2, r1 = bj + dim * nlqj + dim * num2 - 1,
                              r2 = bj + 2 * dim * nlqj + dim * num2 - 3;
                    for (int c = 0; c < 3; ++c)
                    {
                        Kg[r0 + c] += 0.5 * Kl[c][0];
                        Kg[r1 + c] += 0.5 * Kl[c][1];
                        Kg[r2 + c] += 0.5 * Kl[c][2];
                    }
                }
            }
            else
            {
                if (i == j)
                {
                    Kg[base] += Kl[0][0];
                    Kg[base + 1] += Kl[0][1];
                    Kg[base + dim * nlq] += Kl[1][1];
                    JK[base] = dim * (j + 1) - 1;
                    JK[base + 1] = dim * (j + 1);
                    JK[base + dim * nlq] = dim * (j + 1);
                }
                else if (j > i)
                {
                    int num1 = nlq - (nconn - idx);
                    long long r0 = base + dim * num1, r1 = base + dim * nlq + dim * num1 - 1;
                    for (int c = 0; c < 2; ++c)
                    {
                        Kg[r0 + c] += 0.5 * Kl[0][c];
                        Kg[r1 + c] += 0.5 * Kl[1][c];
                        JK[r0 + c] = dim * (j + 1) - 1 + c;
                        JK[r1 + c] = dim * (j + 1) - 1 + c;
                    }
                }
                else
                {
                    int nlqj = p->nlq[j];
                    int num2 = nlqj - ((p->cstart[j + 1] - p->cstart[j]) - conn_pos(p, j, i));
                    long long bj = Kp[j];
                    long long r0 = bj + dim * num2, r1 = bj + dim * nlqj + dim * num2 - 1;
                    for (int c = 0; c < 2; ++c)
                    {
                        Kg[r0 + c] += 0.5 * Kl[c][0];
                        Kg[r1 + c] += 0.5 * Kl[c][1];
                    }
                }
            }
        }
        p->IK[dim * i] = Kp[i] + 1;
        p->IK[dim * i + 1] = Kp[i] + dim * nlq + 1;
        if (dim == 3)
            p->IK[dim * i + 2] = Kp[i] + 2 * dim * nlq;
    }
    p->IK[dim * n] = Kp[n] + 1;
    if (!apply_bc)
        return;

    /* Stiffness::updateStiffnessDispBC (stiffness.h:364-438) */
    double s = 0.0;
    for (int i = 0; i < n; ++i)
    {
        int nlq = p->nlq[i];
        double d0 = Kg[Kp[i]], d1 = Kg[Kp[i] + dim * nlq];
        s += d0 * d0;
        s += d1 * d1;
        if (dim == 3)
        {
            double d2 = Kg[Kp[i] + 2 * dim * nlq - 1];
            s += d2 * d2;
        }
    }
    double norm_diag = sqrt(s);
    for (int i = 0; i < n; ++i)
    {
        int nlq = p->nlq[i];
        for (int k = 0; k < dim; k++)
        {
            if (p->cons[3 * i + k] == 1 || fabs(p->damage_visual[i] - 1.0) < EPS)
            {
                for (int q = p->cstart[i]; q < p->cstart[i + 1]; ++q)
                {
                    int j = p->conns[q];
                    if (j > i)
                        continue;
                    else if (j == i)
                    {
                        if (k == 0)
                        {
                            long long st = (dim == 2) ? Kp[i] : (Kp[i] + 1);
                            for (long long kk = st; kk <= Kp[i] + dim * nlq - 1; kk++)
                                Kg[kk] = 0.0;
                            Kg[Kp[i]] = norm_diag;
                        }
                        else if (k == 1)
                        {
                            Kg[Kp[i] + 1] = 0.0;
                            long long st = (dim == 2) ? (Kp[i] + dim * nlq) : (Kp[i] + dim * nlq + 1);
                            long long en = (dim == 2) ? (Kp[i + 1] - 1) : Kp[i] + 2 * dim * nlq - 2;
                            for (long long kk = st; kk <= en; kk++)
                                Kg[kk] = 0.0;
                            Kg[Kp[i] + dim * nlq] = norm_diag;
                        }
                        else
                        {
                            Kg[Kp[i] + 2] = 0.0;
                            Kg[Kp[i] + dim * nlq + 1] = 0.0;
                            for (long long kk = Kp[i] + 2 * dim * nlq - 1; kk <= Kp[i + 1] - 1; kk++)
                                Kg[kk] = 0.0;
                            Kg[Kp[i] + 2 * dim * nlq - 1] = norm_diag;
                        }
                    }
                    else
                    {
                        int nlqj = p->nlq[j];
                        int num2 = nlqj - ((p->cstart[j + 1] - p->cstart[j]) - conn_pos(p, j, i));
                        Kg[Kp[j] + dim * num2 + k] = 0;
                        Kg[Kp[j] + dim * nlqj + dim * num2 - 1 + k] = 0;
                        if (dim == 3)
                            Kg[Kp[j] + 2 * dim * nlqj + dim * num2 - 3 + k] = 0;
                    }
                }
                p->residual[dim * i + k] = 0.0;
            }
        }
    }
}

void lpmo_export_csr(const lpmo_problem *p, long long *K_pointer, long long *IK, long long *JK, double *K)
{
    const int n = p->n, dim = p->dim;
    const long long nnz = p->K_pointer[n];
    if (K_pointer)
        memcpy(K_pointer, p->K_pointer, sizeof(long long) * (n + 1));
    if (IK)
        memcpy(IK, p->IK, sizeof(long long) * ((size_t)dim * n + 1));
    if (JK)
        memcpy(JK, p->JK, sizeof(long long) * nnz);
    if (K)
        memcpy(K, p->K, sizeof(double) * nnz);
}

/* Solver::LPM_CG (solver.h:277-354) with the RCI CG semantics of the shim: x0 = 0,
 * ||r||^2 <= rtol * ||r0||^2 + atol, iteration cap ipar[4] = problem size. */
long long lpmo_cg(lpmo_problem *p, double *disp)
{
    const int dim = p->dim;
    const long long n = (long long)dim * p->n;
    const long long *Kp = p->K_pointer;
    /* full symmetric CSR from the 1-based upper CSR: lower entries first (by source row), then upper */
    long long *cnt = (long long *)calloc(n + 1, sizeof(long long));
    for (long long r = 0; r < n; ++r)
        for (long long q = p->IK[r] - 1; q < p->IK[r + 1] - 1; ++q)
        {
            long long c = p->JK[q] - 1;
            cnt[r]++;
            if (c != r)
                cnt[c]++;
        }
    long long *rp = (long long *)calloc(n + 1, sizeof(long long));
    for (long long r = 0; r < n; ++r)
        rp[r + 1] = rp[r] + cnt[r];
    long long *ci = (long long *)malloc(sizeof(long long) * (rp[n] + 1));
    double *v = (double *)malloc(sizeof(double) * (rp[n] + 1));
    long long *fill = (long long *)malloc(sizeof(long long) * (n + 1));
    memcpy(fill, rp, sizeof(long long) * n);
    for (long long r = 0; r < n; ++r)
        for (long long q = p->IK[r] - 1; q < p->IK[r + 1] - 1; ++q)
        {
            long long c = p->JK[q] - 1;
            if (c != r)
            {
                ci[fill[c]] = r;
                v[fill[c]++] = p->K[q];
            }
        }
    for (long long r = 0; r < n; ++r)
        for (long long q = p->IK[r] - 1; q < p->IK[r + 1] - 1; ++q)
        {
            ci[fill[r]] = p->JK[q] - 1;
            v[fill[r]++] = p->K[q];
        }
    (void)Kp;
    double *r = (double *)malloc(sizeof(double) * n), *pp = (double *)malloc(sizeof(double) * n),
           *Ap = (double *)malloc(sizeof(double) * n);
    for (long long q = 0; q < n; ++q)
    {
        disp[q] = 0;
        r[q] = p->residual[q];
        pp[q] = r[q];
    }
    double rr = 0.0;
    for (long long q = 0; q < n; ++q)
        rr += r[q] * r[q];
    const double stop = p->cg_rtol * rr + p->cg_atol;
    long long maxit = (p->cg_maxit > 0) ? p->cg_maxit : n;
    long long it = 0;
    if (!(rr <= stop))
    {
        while (1)
        {
            for (long long row = 0; row < n; ++row)
            {
                double s = 0.0;
                for (long long q = rp[row]; q < rp[row + 1]; ++q)
                    s += v[q] * pp[ci[q]];
                Ap[row] = 1.0 * s;
            }
            double pAp = 0.0;
            for (long long q = 0; q < n; ++q)
                pAp += pp[q] * Ap[q];
            if (pAp == 0.0)
                break;
            double alpha = rr / pAp;
            for (long long q = 0; q < n; ++q)
            {
                disp[q] += alpha * pp[q];
                r[q] -= alpha * Ap[q];
            }
            it++;
            double rn = 0.0;
            for (long long q = 0; q < n; ++q)
                rn += r[q] * r[q];
            if (rn <= stop || it >= maxit)
                break;
            double beta = rn / rr;
            rr = rn;
            for (long long q = 0; q < n; ++q)
                pp[q] = r[q] + beta * pp[q];
        }
    }
    free(cnt);
    free(rp);
    free(ci);
    free(v);
    free(fill);
    free(r);
    free(pp);
    free(Ap);
    return it;
}

/* ------------------------------------------------------------- load stepping */
/* Solver::updateForceBC (solver.h:167-188) then Solver::updateDisplacementBC (solver.h:129-164),
 * Relative mode */
void lpmo_apply_bc(lpmo_problem *p, const lpmo_loadstep *s)
{
    for (int f = 0; f < s->nforce; ++f)
    {
        const lpmo_forcebc *bc = s->force + f;
        int num = bc->count;
        for (int q = 0; q < num; ++q)
        {
            int i = bc->ids[q];
            p->pex[3 * i] += bc->fx / num;
            p->pex[3 * i + 1] += bc->fy / num;
            p->pex[3 * i + 2] += bc->fz / num;
        }
    }
    for (int d = 0; d < s->ndisp; ++d)
    {
        const lpmo_dispbc *bc = s->disp + d;
        for (int q = 0; q < bc->count; ++q)
        {
            int i = bc->ids[q];
            double dx[3] = {0, 0, 0};
            dx[bc->flag] = bc->step;
            for (int k = 0; k < 3; ++k)
                p->xyz[3 * i + k] = p->xyz[3 * i + k] + dx[k];
            p->cons[3 * i + bc->flag] = 1;
        }
    }
}

/* Solver::NewtonIteration (solver.h:55-90) */
static int newton(lpmo_problem *p, lpmo_stats *st)
{
    const int dim = p->dim;
    lpmo_update_geometry(p);
    lpmo_update_force_state(p);
    double nres = lpmo_update_rr(p);
    double nreac = sqrt(p->reaction_sq);
    double tol_mult = (nres < nreac) ? nreac : nres; /* std::max */
    int ni = 0;
    double *disp = (double *)malloc(sizeof(double) * dim * p->n + 8);
    while (nres > p->tol * tol_mult)
    {
        if (++ni > p->max_iter)
        {
            free(disp);
            return p->max_iter;
        }
        if (p->tangent)
            lpmo_assemble(p, 1);
        long long it = lpmo_cg(p, disp);
        if (st)
        {
            st->newton_solves++;
            st->cg_iters += it;
        }
        /* Solver::solveLinearSystem position update (solver.h:101-108) */
        for (int i = 0; i < p->n; ++i)
        {
            double dx[3] = {0, 0, 0};
            for (int k = 0; k < dim; ++k)
                dx[k] += disp[dim * i + k];
            for (int k = 0; k < 3; ++k)
                p->xyz[3 * i + k] = p->xyz[3 * i + k] + dx[k];
        }
        lpmo_update_geometry(p);
        lpmo_update_force_state(p);
        nres = lpmo_update_rr(p);
    }
    free(disp);
    return ni;
}

/* the nonlocal damage rate of SolverStatic::updateStaticDamage (solver_static.h:35-52) and
 * SolverFatigue::updateFatigueDamage (solver_fatigue.h:79-115), with func_phi (lpm.h:48-52) */
static void nonlocal_rate(lpmo_problem *p)
{
    const int n = p->n;
    for (int i = 0; i < n; ++i)
    {
        if (p->type[i] == p->undamaged_type)
            continue;
        double A = 0;
        p->ddot_nonlocal[i] = 0;
        for (int q = p->nlstart[i]; q < p->nlstart[i + 1]; ++q)
        {
            int j = p->nlist[q];
            if (p->type[j] == p->undamaged_type)
                continue;
            double ds = dist(p->xyz + 3 * i, p->xyz + 3 * j);
            double V_m = p->pvol * p->nb[j] / p->nneighbors;
            double phi = pow(1 / (1 + pow(ds / p->nonlocal_L, 8)), 2);
            p->ddot_nonlocal[i] += p->ddot_local[j] * phi * V_m;
            A += pow(1 / (1 + pow(ds / p->nonlocal_L, 8)), 2) * V_m;
        }
        p->ddot_nonlocal[i] /= A;
    }
}

/* SolverStatic::updateStaticDamage (solver_static.h:32-62) */
static int update_static_damage(lpmo_problem *p)
{
    const int n = p->n;
    nonlocal_rate(p);
    int any = 0;
    for (int i = 0; i < n; ++i)
    {
        if (p->type[i] == p->undamaged_type)
            continue;
        int changed = 0;
        if (p->ptype == LPMO_J2 || p->ptype == LPMO_ELASTIC_DAMAGE)
        {
            /* ParticleJ2Plasticity::updateParticleStaticDamage (particle_j2plasticity.h:142-152),
             * ParticleElasticDamage::updateParticleStaticDamage (particle_elastic_damage.h:172-181) */
            p->damage[i] += p->ddot_nonlocal[i];
            if (p->damage[i] >= p->damage_threshold)
                p->damage[i] = 1;
            changed = fabs(p->damage[i] - p->damage_last[i]) > 1e-3;
        }
        else if (p->ptype == LPMO_ELASTIC)
        {
            /* ParticleElastic::updateParticleStaticDamage (particle_elastic.h:52-68); fatigue
             * particles keep Particle::updateParticleStaticDamage, which changes nothing
             * (particle.h:63) */
            for (int b = B0(p, i); b < BE(p, i); ++b)
                if (p->bstrain[b] >= p->critical_bstrain && fabs(p->bdamage[b] - 1.0) > EPS)
                {
                    changed = 1;
                    p->bdamage[b] = 1;
                }
        }
        any = changed || any;
    }
    return any;
}

/* Assembly::storeStateVar (assembly.h:141-148) */
static void store_state(lpmo_problem *p)
{
    memcpy(p->xyz_last, p->xyz, sizeof(double) * 3 * p->n);
    memcpy(p->damage_last, p->damage, sizeof(double) * p->n);
    memcpy(p->sv_last, p->sv, sizeof(double) * p->nsv * p->n);
    memcpy(p->dis_last, p->dis, sizeof(double) * p->nbonds);
    memcpy(p->bdamage_last, p->bdamage, sizeof(double) * p->nbonds);
    memcpy(p->bforce_last, p->bforce, sizeof(double) * p->nbonds);
    memcpy(p->dLp_last, p->dLp, sizeof(double) * p->nbonds);
}

/* Assembly::resetStateVar(true) (assembly.h:151-159) */
static void reset_state(lpmo_problem *p)
{
    memcpy(p->xyz, p->xyz_last, sizeof(double) * 3 * p->n);
    memcpy(p->damage, p->damage_last, sizeof(double) * p->n);
    memcpy(p->sv, p->sv_last, sizeof(double) * p->nsv * p->n);
    memcpy(p->dis, p->dis_last, sizeof(double) * p->nbonds);
    memcpy(p->bdamage, p->bdamage_last, sizeof(double) * p->nbonds);
    memcpy(p->bforce, p->bforce_last, sizeof(double) * p->nbonds);
    memcpy(p->dLp, p->dLp_last, sizeof(double) * p->nbonds);
}

/* SolverStatic::solveProblemStep (solver_static.h:99-152) */
int lpmo_solve_problem_step(lpmo_problem *p, const lpmo_loadstep *s, lpmo_stats *st)
{
    lpmo_apply_bc(p, s);
    int n_newton = 0, new_damaged = 0;
    do
    {
        if (!p->tangent)
            lpmo_assemble(p, 1);
        n_newton = newton(p, st);
        if (n_newton >= p->max_iter)
            break;
        lpmo_update_state_var(p);
        new_damaged = update_static_damage(p);
        store_state(p);
        if (new_damaged)
        {
            lpmo_update_geometry(p);
            lpmo_update_force_state(p);
        }
    } while (new_damaged);
    return n_newton < p->max_iter;
}

/* one load step of SolverStatic::solveProblem (solver_static.h:72-93): on failure reset the
 * state, halve the step, run the two halves (each of which may be halved again) */
static int solve_rec(lpmo_problem *p, const lpmo_loadstep *s, double scale, lpmo_stats *st, int depth)
{
    lpmo_dispbc db[64];
    lpmo_forcebc fb[64];
    lpmo_loadstep sc = *s;
    if (s->ndisp > 64 || s->nforce > 64)
        return 0;
    for (int d = 0; d < s->ndisp; ++d)
    {
        db[d] = s->disp[d];
        db[d].step = s->disp[d].step * scale;
    }
    for (int f = 0; f < s->nforce; ++f)
    {
        fb[f] = s->force[f];
        fb[f].fx = s->force[f].fx * scale;
        fb[f].fy = s->force[f].fy * scale;
        fb[f].fz = s->force[f].fz * scale;
    }
    sc.disp = db;
    sc.force = fb;
    if (lpmo_solve_problem_step(p, &sc, st))
        return 1;
    if (depth >= 30)
        return 0;
    reset_state(p);
    if (st)
        st->cuts++;
    return solve_rec(p, s, scale / 2.0, st, depth + 1) && solve_rec(p, s, scale / 2.0, st, depth + 1);
}

int lpmo_solve_load_step(lpmo_problem *p, const lpmo_loadstep *s, lpmo_stats *st)
{
    if (st)
        memset(st, 0, sizeof *st);
    int ok = solve_rec(p, s, 1.0, st, 0);
    if (st)
    {
        st->converged = ok;
        st->reaction_norm = sqrt(p->reaction_sq);
    }
    return ok;
}

void lpmo_read_state(const lpmo_problem *p, double *xyz, double *pin, double *stress, double *damage,
                     double *damage_visual, double *state_var, double *bdamage)
{
    const int n = p->n;
    if (xyz) memcpy(xyz, p->xyz, sizeof(double) * 3 * n);
    if (pin) memcpy(pin, p->pin, sizeof(double) * 3 * n);
    if (stress) memcpy(stress, p->stress, sizeof(double) * 6 * n);
    if (damage) memcpy(damage, p->damage, sizeof(double) * n);
    if (damage_visual) memcpy(damage_visual, p->damage_visual, sizeof(double) * n);
    if (state_var) memcpy(state_var, p->sv, sizeof(double) * p->nsv * n);
    if (bdamage) memcpy(bdamage, p->bdamage, sizeof(double) * p->nbonds);
}

void lpmo_set_xyz(lpmo_problem *p, const double *xyz)
{
    memcpy(p->xyz, xyz, sizeof(double) * 3 * p->n);
}

void lpmo_get_bond_kntv(const lpmo_problem *p, double *kn, double *tv)
{
    memcpy(kn, p->Kn, sizeof(double) * p->nbonds);
    memcpy(tv, p->Tv, sizeof(double) * p->nbonds);
}

void lpmo_set_bond_kntv(lpmo_problem *p, const double *kn, const double *tv)
{
    memcpy(p->Kn, kn, sizeof(double) * p->nbonds);
    memcpy(p->Tv, tv, sizeof(double) * p->nbonds);
}

void lpmo_set_bond_damage(lpmo_problem *p, const double *bdamage)
{
    memcpy(p->bdamage, bdamage, sizeof(double) * p->nbonds);
    memcpy(p->bdamage_last, bdamage, sizeof(double) * p->nbonds);
}

/* ------------------------------------------------------------------ SolverFatigue (solver_fatigue.h) */

/* SolverFatigue::solveProblemStep (solver_fatigue.h:278-302): BCs, the stiffness from the
 * current state, Newton; no damage loop */
int lpmo_fatigue_solve_step(lpmo_problem *p, const lpmo_loadstep *s, lpmo_stats *st)
{
    lpmo_apply_bc(p, s);
    if (!p->tangent)
        lpmo_assemble(p, 1);
    const int n_newton = newton(p, st);
    if (st)
        st->reaction_norm = sqrt(p->reaction_sq);
    return n_newton < p->max_iter;
}

/* SolverFatigue::updateFatigueDamage (solver_fatigue.h:76-126) with
 * ParticleFatigueHCF::updateParticleFatigueDamage (particle_fatigue_hcf.h:148-160); the other
 * particle types keep Particle::updateParticleFatigueDamage, which changes nothing
 * (particle.h:64) */
int lpmo_fatigue_update_damage(lpmo_problem *p, double dNdt)
{
    nonlocal_rate(p);
    int any = 0;
    for (int i = 0; i < p->n; ++i)
    {
        if (p->type[i] == p->undamaged_type)
            continue;
        int changed = 0;
        if (p->ptype == LPMO_FATIGUE_HCF)
        {
            p->damage[i] += p->ddot_nonlocal[i] * dNdt;
            if (p->damage[i] >= p->damage_threshold)
                p->damage[i] = 1;
            p->sv[3 * i + 1] = 2147483647.0; /* INT_MAX */
            p->sv[3 * i + 2] = 0;
            changed = fabs(p->damage[i] - p->damage_last[i]) > 1e-3;
        }
        any = changed || any;
    }
    return any;
}

/* SolverFatigue::solveProblemOneCycle (solver_fatigue.h:221-241) */
int lpmo_fatigue_cycle(lpmo_problem *p, const lpmo_loadstep *steps, int nsteps, double dNdt, lpmo_stats *st)
{
    if (st)
        memset(st, 0, sizeof *st);
    int all_converged = 1;
    for (int k = 0; k < nsteps; ++k)
    {
        /* the reference ignores a step that did not converge (is_converged is unused) */
        if (!lpmo_fatigue_solve_step(p, &steps[k], st))
        {
            all_converged = 0;
            if (st)
                st->cuts++;
        }
        lpmo_update_state_var(p);
    }
    const int any = lpmo_fatigue_update_damage(p, dNdt);
    store_state(p);
    lpmo_update_geometry(p);
    lpmo_update_force_state(p);
    if (st)
    {
        st->converged = all_converged;
        st->reaction_norm = sqrt(p->reaction_sq);
    }
    return any;
}

/* one load step of SolverFatigue::solveProblemStatic (solver_fatigue.h:244-275): on failure reset
 * the state, halve the step and run the two halves; every converged (sub)step is followed by
 * updateStateVar and storeStateVar */
static int fatigue_static_rec(lpmo_problem *p, const lpmo_loadstep *s, double scale, lpmo_stats *st, int depth)
{
    lpmo_dispbc db[64];
    lpmo_forcebc fb[64];
    lpmo_loadstep sc = *s;
    if (s->ndisp > 64 || s->nforce > 64)
        return 0;
    for (int d = 0; d < s->ndisp; ++d)
    {
        db[d] = s->disp[d];
        db[d].step = s->disp[d].step * scale;
    }
    for (int f = 0; f < s->nforce; ++f)
    {
        fb[f] = s->force[f];
        fb[f].fx = s->force[f].fx * scale;
        fb[f].fy = s->force[f].fy * scale;
        fb[f].fz = s->force[f].fz * scale;
    }
    sc.disp = db;
    sc.force = fb;
    if (lpmo_fatigue_solve_step(p, &sc, st))
    {
        lpmo_update_state_var(p);
        store_state(p);
        return 1;
    }
    if (depth >= 30)
        return 0;
    reset_state(p);
    if (st)
        st->cuts++;
    return fatigue_static_rec(p, s, scale / 2.0, st, depth + 1) &&
           fatigue_static_rec(p, s, scale / 2.0, st, depth + 1);
}

int lpmo_fatigue_static_step(lpmo_problem *p, const lpmo_loadstep *s, lpmo_stats *st)
{
    if (st)
        memset(st, 0, sizeof *st);
    const int ok = fatigue_static_rec(p, s, 1.0, st, 0);
    if (st)
    {
        st->converged = ok;
        st->reaction_norm = sqrt(p->reaction_sq);
    }
    return ok;
}
