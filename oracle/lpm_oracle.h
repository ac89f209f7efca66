/*
 * Test infrastructure (oracle): a plain-C, single-threaded restatement of the LPM-CPP
 * implicit quasi-static step.  It is the checker for the device path: only tests, the smoke
 * check and the CPU-baseline leg of the benchmark load it.  Each function names the
 * reference file:line it follows.  Built by oracle/Makefile into oracle/liblpm_oracle.so.
 */
#ifndef LPM_ORACLE_H
#define LPM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* LatticeType order of include/lpm.h:97-106 */
enum { LPMO_SQUARE2D = 0, LPMO_HEXAGON2D = 1, LPMO_SC3D = 2, LPMO_FCC3D = 3, LPMO_BCC3D = 4 };
/* ParticleType order of include/lpm.h:89-95 */
enum { LPMO_ELASTIC = 0, LPMO_ELASTIC_DAMAGE = 1, LPMO_J2 = 2, LPMO_FATIGUE_HCF = 3 };

typedef struct
{
    int lattice;
    int ptype;
    int n;                 /* particles */
    const double *xyz;     /* n*3, generation order == particle id */
    const int *type;       /* n, or NULL (all 0) */
    double radius;
    int plane_stress;
    double E, mu, critical_bstrain;
    double sigmay, xi, H, A; /* J2 only */
    double nonlocal_L;
    double nonlocal_cutoff_ratio; /* > 0: run the nonlocal neighbour search (assembly.h:118-130) */
    int undamaged_type;
    int max_iter;
    double tol_iter;
    double cg_rtol, cg_atol;   /* squared-norm tolerances of the RCI CG (solver.h:312-313) */
    long long cg_maxit;        /* 0 -> problem size (solver.h:308) */
    /* optional bond lists in place of the search: per particle nb0[i] layer-0 partners then
     * nb1[i] layer-1 partners, concatenated in p2 (Assembly(dumpFile, bondFile, ...) and
     * Assembly::readBond, assembly.h:84-95, 391-424); NULL -> Assembly::createBonds */
    const int *bond_nb0, *bond_nb1, *bond_p2;
    /* 1: tangent mode, the stiffness re-assembled from the current state before every Newton
     * solve (no assembly at the start of a damage iteration); 0: K fixed per load step as in
     * SolverStatic::solveProblemStep (solver_static.h:107-118) */
    int tangent;
    /* ParticleElasticDamage only (setParticleProperty, particle_elastic_damage.h:183-220) */
    double k0, k1, comp_tensile_ratio, damage_threshold;
    /* ParticleFatigueHCF only (setParticleProperty, particle_fatigue_hcf.h:163-205): the damage
     * rate A * pow(max energy, B) * pow(energy range, d); damage_threshold above is its p_d_thres.
     * The fatigue limit ratio is stored by the reference but unused (calcEqEnergy returns the
     * total energy, particle_fatigue_hcf.h:123). */
    double fatigue_A, fatigue_B, fatigue_d, fatigue_limit_ratio;
    /* C11 > 0: the (C11, C12, C44) overloads of setParticleProperty (particle_elastic.h:110-140,
     * particle_elastic_damage.h:218-250) in place of E, mu and plane_stress (not for J2) */
    double C11, C12, C44;
} lpmo_desc;

typedef struct
{
    const int *ids;
    int count;
    int flag;   /* 0 'x', 1 'y', 2 'z' */
    double step;
} lpmo_dispbc;

typedef struct
{
    const int *ids;
    int count;
    double fx, fy, fz;
} lpmo_forcebc;

typedef struct
{
    const lpmo_dispbc *disp;
    int ndisp;
    const lpmo_forcebc *force;
    int nforce;
} lpmo_loadstep;

typedef struct
{
    int newton_solves;     /* linear solves (Newton iterations that ran CG) */
    long long cg_iters;
    int cuts;              /* load-step halvings */
    int converged;
    double reaction_norm;  /* ||all reaction history|| */
} lpmo_stats;

typedef struct lpmo_problem lpmo_problem;

/* utilities.h:15-91 */
void lpmo_rmatrix(int eulerflag, const double angles[3], double R[9]);
/* utilities.h:93-310 (+ a BCC generator, which the reference lacks); returns the count,
 * writes at most cap points (n*3 doubles) when out != NULL */
long lpmo_generate(int lattice, double radius, const double box[6], const double R[9], double *out, long cap);

lpmo_problem *lpmo_create(const lpmo_desc *d);
void lpmo_destroy(lpmo_problem *p);

int lpmo_dim(const lpmo_problem *p);
long lpmo_nbonds(const lpmo_problem *p);
long lpmo_nconn_total(const lpmo_problem *p);
long long lpmo_nnz_upper(const lpmo_problem *p);
/* nb0/nb1: n each; p2: nbonds (per particle: layer-0 list then layer-1 list) */
void lpmo_get_bonds(const lpmo_problem *p, int *nb0, int *nb1, int *p2);
/* nconn/nlq: n each; conns: nconn_total */
void lpmo_get_conns(const lpmo_problem *p, int *nconn, int *nlq, int *conns);

/* assembly.h:133-138 then assembly.h:179-191 */
void lpmo_update_geometry(lpmo_problem *p);
void lpmo_update_force_state(lpmo_problem *p);
void lpmo_update_state_var(lpmo_problem *p);
/* solver.h:112-126; returns ||residual||, appends the reaction history */
double lpmo_update_rr(lpmo_problem *p);

/* stiffness.h:74-89 + 198-361 + 364-438: reference layout, 1-based upper CSR */
void lpmo_assemble(lpmo_problem *p, int apply_bc);
void lpmo_export_csr(const lpmo_problem *p, long long *K_pointer, long long *IK, long long *JK, double *K);
/* solver.h:277-354 on the current K and residual; returns CG iterations, disp (n*dim) out */
long long lpmo_cg(lpmo_problem *p, double *disp);

/* solver.h:167-188 / 129-164 */
void lpmo_apply_bc(lpmo_problem *p, const lpmo_loadstep *s);
/* solver_static.h:99-152; returns 1 when converged */
int lpmo_solve_problem_step(lpmo_problem *p, const lpmo_loadstep *s, lpmo_stats *st);
/* one entry of solver_static.h:72-93: solve, and on failure reset, halve, retry */
int lpmo_solve_load_step(lpmo_problem *p, const lpmo_loadstep *s, lpmo_stats *st);

/* SolverFatigue (include/solver_fatigue.h).  One fatigue step: updateForceBC,
 * updateDisplacementBC, the stiffness from the current state, NewtonIteration; no damage loop
 * (solver_fatigue.h:278-302).  Returns 1 when Newton converged. */
int lpmo_fatigue_solve_step(lpmo_problem *p, const lpmo_loadstep *s, lpmo_stats *st);
/* SolverFatigue::updateFatigueDamage (solver_fatigue.h:76-126): the nonlocal average of the
 * local rates, then damage += rate * dNdt per damageable particle; returns any_damaged */
int lpmo_fatigue_update_damage(lpmo_problem *p, double dNdt);
/* SolverFatigue::solveProblemOneCycle (solver_fatigue.h:221-241): every step of the cycle
 * (fatigue step + updateStateVar, failures ignored as in the reference), then
 * updateFatigueDamage(dNdt), storeStateVar, updateGeometry, updateForceState.  Returns
 * updateFatigueDamage's flag; st sums the steps' Newton solves and counts unconverged steps
 * in st->cuts. */
int lpmo_fatigue_cycle(lpmo_problem *p, const lpmo_loadstep *steps, int nsteps, double dNdt, lpmo_stats *st);
/* one entry of SolverFatigue::solveProblemStatic (solver_fatigue.h:244-275): the fatigue step,
 * on failure reset, halve and retry; after each converged (sub)step updateStateVar and
 * storeStateVar.  Returns 1 when every (sub)step converged. */
int lpmo_fatigue_static_step(lpmo_problem *p, const lpmo_loadstep *s, lpmo_stats *st);

/* state read-back (n*3 / n*6 / n / n*nsv / nbonds) */
void lpmo_read_state(const lpmo_problem *p, double *xyz, double *pin, double *stress, double *damage,
                     double *damage_visual, double *state_var, double *bdamage);
int lpmo_nstate_var(const lpmo_problem *p);
void lpmo_read_residual(const lpmo_problem *p, double *res);
void lpmo_set_xyz(lpmo_problem *p, const double *xyz);
/* per-bond coefficients and damage, in bond order (owner, layer 0 then layer 1).  An LPM-CPP
 * example sets them by writing Bond::Kn / Tv / bdamage (bond.h:25-27) after setParticleProperty
 * and before the first updateForceState: a heterogeneous material or a pre-crack.  Setting the
 * damage also sets bdamage_last, so resetStateVar(true) (particle.h:141) restores it. */
void lpmo_get_bond_kntv(const lpmo_problem *p, double *kn, double *tv);
void lpmo_set_bond_kntv(lpmo_problem *p, const double *kn, const double *tv);
void lpmo_set_bond_damage(lpmo_problem *p, const double *bdamage);

#ifdef __cplusplus
}
#endif
#endif
