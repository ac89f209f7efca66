/*
 * lpmgpu: B200-native implicit quasi-static step of the nonlocal lattice particle method.
 *
 * This is the C ABI of liblpmgpu.so: plain pointers, sizes and status codes, no CUDA or
 * torch types.  It replaces, for one load step of LPM-CPP, the code path
 *   SolverStatic<nlayer>::solveProblem / solveProblemStep   (include/solver_static.h:65-152)
 *   Solver<nlayer>::NewtonIteration / updateRR / BCs / LPM_CG (include/solver.h:55-188, 277-354)
 *   Stiffness<nlayer>::calcStiffness2D/3D / updateStiffnessDispBC (include/stiffness.h:198-438)
 *   Assembly<nlayer>::createBonds / updateConnections / updateGeometry / updateForceState
 *                                                            (include/assembly.h:133-266)
 * (paths inside the LPM-CPP tree).  Every entry point returns an lpmgpu_status; none exits
 * the process.  One handle belongs to one host thread at a time; the server API is the
 * thread-safe entry for concurrent submitters.
 */
#ifndef LPMGPU_H
#define LPMGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------------------- status */
typedef enum
{
    LPMGPU_OK = 0,
    LPMGPU_ERR_INVALID_ARG = 1,   /* bad pointer, size or enum value */
    LPMGPU_ERR_CUDA = 2,          /* a CUDA runtime call failed (message via lpmgpu_last_error) */
    LPMGPU_ERR_OUT_OF_MEMORY = 3, /* device allocation failed */
    LPMGPU_ERR_NEWTON = 4,        /* Newton hit max_iter (solver_static.h:122, the load-cut trigger) */
    LPMGPU_ERR_CG_MAXIT = 5,      /* a CG solve reached its cap; printed and ignored by the reference
                                     (solver.h:338-349); the handle entry points report it through
                                     stats, only lpmgpu_cg_bsr_noalloc returns it */
    LPMGPU_ERR_TIMEOUT = 6,       /* a bounded device-side wait gave up; the context stays usable */
    LPMGPU_ERR_TOPOLOGY = 7,      /* a particle without bonds, or more bonds/connections than supported */
    LPMGPU_ERR_BUDGET = 8,        /* request larger than the server's HBM budget */
    LPMGPU_ERR_CUTS = 9,          /* a load step was halved more than 30 times */
    LPMGPU_ERR_NOT_READY = 10,    /* server: result not available yet */
    LPMGPU_ERR_NO_DEVICE = 11,    /* no CUDA device; the library has no CPU fallback */
    LPMGPU_ERR_NOT_SPD = 12,      /* direct solve: the stiffness is not positive definite */
    LPMGPU_ERR_CG_BREAKDOWN = 13  /* lpmgpu_cg_bsr_noalloc: p.Ap == 0 (singular or indefinite matrix) */
} lpmgpu_status;

/* LatticeType (include/lpm.h:97-106); BCC3D covers the three BCC enum values */
enum { LPMGPU_SQUARE2D = 0, LPMGPU_HEXAGON2D = 1, LPMGPU_SC3D = 2, LPMGPU_FCC3D = 3, LPMGPU_BCC3D = 4 };
/* ParticleType (include/lpm.h:89-95) values on this path */
enum { LPMGPU_ELASTIC = 0, LPMGPU_ELASTIC_DAMAGE = 1, LPMGPU_J2 = 2, LPMGPU_FATIGUE_HCF = 3 };
/* linear-solve precision */
enum { LPMGPU_FP64 = 0, LPMGPU_MIXED = 1 };

typedef struct lpmgpu_solver lpmgpu_solver;

/* One problem (an Assembly plus its solver settings). */
typedef struct
{
    int32_t lattice;         /* LPMGPU_SQUARE2D .. LPMGPU_BCC3D */
    int32_t ptype;           /* LPMGPU_ELASTIC, LPMGPU_ELASTIC_DAMAGE, LPMGPU_J2 or LPMGPU_FATIGUE_HCF */
    int32_t n;               /* particles */
    const double *xyz;       /* host, n*3; row q is particle id q (generation order) */
    const int32_t *type;     /* host, n particle types, or NULL for all 0 */
    double radius;           /* UnitCell radius */
    int32_t plane_stress;    /* setParticleProperty is_plane_stress */
    double E, mu;            /* Young's modulus, Poisson's ratio */
    double critical_bstrain; /* elastic bond breaking strain (particle_elastic.h:60) */
    double sigmay, xi, H, A; /* J2 parameters (particle_j2plasticity.h:155-163) */
    double nonlocal_L;       /* Particle::nonlocal_L, the length of the nonlocal damage weight */
    int32_t undamaged_type;  /* SolverStatic undamaged_pt_type */
    int32_t max_iter;        /* Newton iteration cap (max_NR_iter) */
    double tol_iter;         /* Newton tolerance (tol_NR_iter) */
    double cg_rtol, cg_atol; /* squared-norm CG test ||r||^2 <= rtol*||r0||^2 + atol (solver.h:312-313) */
    int64_t cg_maxit;        /* CG cap, 0 = problem size (solver.h:308) */
    int32_t precision;       /* LPMGPU_FP64 or LPMGPU_MIXED */
    int32_t device;          /* CUDA device ordinal */
    /* Optional inputs (NULL = derive them as the reference's Assembly constructor would).
     * bond_nb0/bond_nb1/bond_p2: the bond lists (per particle its layer-0 partners then its
     * layer-1 partners), e.g. from Assembly::readBond (assembly.h:391-424) or with bonds left
     * out along a pre-crack; every bond needs its opposite.  bond_kn/bond_tv: per-bond
     * coefficients in the same order (what setParticleProperty stored), overriding E/mu.
     * bond_damage: initial bond damage in the same order (1 = broken). */
    const int32_t *bond_nb0, *bond_nb1, *bond_p2;
    const double *bond_kn, *bond_tv, *bond_damage;
    /* 1: tangent mode: K is re-assembled from the current state before every Newton linear
     * solve (and not at the start of a damage iteration).  0: K fixed per load step, as in
     * SolverStatic::solveProblemStep (solver_static.h:107-118).  No counterpart in
     * SolverStatic; its Newton loop and assembly calls are those of solver.h:55-90 and
     * stiffness.h, re-ordered. */
    int32_t tangent;
    /* > 0: Assembly::searchNonlocalNeighbors(nonlocal_cutoff_ratio) (assembly.h:118-130) runs on the
     * device at creation, and SolverStatic::updateStaticDamage (solver_static.h:32-62) averages the
     * local damage rates over those neighbours.  0: no search; the nonlocal rate is then 0/0 as in
     * the reference without the search. */
    double nonlocal_cutoff_ratio;
    /* LPMGPU_ELASTIC_DAMAGE (ParticleElasticDamage::setParticleProperty,
     * particle_elastic_damage.h:183-220): damage surface k0 + k1 D on the strain energy density,
     * the compression/tension ratio of its equivalent strain, and the damage threshold */
    double k0, k1, comp_tensile_ratio, damage_threshold;
    /* LPMGPU_FATIGUE_HCF (ParticleFatigueHCF::setParticleProperty, particle_fatigue_hcf.h:163-205):
     * the damage rate fatigue_A * pow(largest energy, fatigue_B) * pow(energy range of the cycle,
     * fatigue_d); damage_threshold above is its damage threshold.  fatigue_limit_ratio is kept for
     * the interface but, as in the reference, does not enter the result (calcEqEnergy returns the
     * total energy, particle_fatigue_hcf.h:123). */
    double fatigue_A, fatigue_B, fatigue_d, fatigue_limit_ratio;
    /* Optional nonlocal neighbour lists in place of the search (NULL = none given): particle i's
     * list is nonlocal_count[i] ids, the lists concatenated in nonlocal_ids, each in the order of
     * Particle::neighbors_nonlocal (particle.h:37), which the averaging sums in.  An Assembly on
     * which searchNonlocalNeighbors ran (assembly.h:118-130) holds them.  Not together with
     * nonlocal_cutoff_ratio > 0. */
    const int32_t *nonlocal_count, *nonlocal_ids;
    /* Linear solver of the Newton iterations.  0: the CG (Solver::LPM_CG).  1: the direct band
     * Cholesky (lpmgpu_solve_direct; Solver::LPM_PARDISO's role, solver.h:191-274).  2: the CG
     * first, and the band Cholesky only for a system the CG could not solve (cap reached or
     * p.Ap == 0) while its band fits (at most 32 GiB); the C++ and Python drop-ins use 2, with
     * the CG's squared-norm test at 1e-24, for SolverMode::PARDISO.  The direct solve is FP64
     * whatever the precision. */
    int32_t direct;
    /* C11 > 0: the bond coefficients come from these elastic constants, as the (C11, C12, C44)
     * overloads of setParticleProperty set them (particle_elastic.h:110-140,
     * particle_elastic_damage.h:218-250), in place of E, mu and plane_stress; for elastic and
     * elastic-damage particles (J2 keeps E and mu for its return map). */
    double C11, C12, C44;
} lpmgpu_desc;

/* Displacement / force boundary condition of one load step (boundary.h:10-44, Relative mode). */
typedef struct
{
    const int32_t *ids; /* host particle ids of the group */
    int32_t count;
    int32_t flag;       /* 0 'x', 1 'y', 2 'z' */
    double step;
} lpmgpu_dispbc;

typedef struct
{
    const int32_t *ids;
    int32_t count;
    double fx, fy, fz;
} lpmgpu_forcebc;

typedef struct
{
    const lpmgpu_dispbc *disp;
    int32_t ndisp;
    const lpmgpu_forcebc *force;
    int32_t nforce;
} lpmgpu_load_step;

typedef struct
{
    int32_t converged;       /* 1 when the load step (with any halvings) converged */
    int32_t newton_solves;   /* linear solves (Newton iterations that ran CG) */
    int32_t cuts;            /* load-step halvings (solver_static.h:78-87) */
    int32_t damage_iters;    /* passes of the damage loop (solver_static.h:107-139) */
    int64_t cg_iters;        /* CG iterations (FP32 inner + FP64 in mixed mode) */
    int64_t cg_maxit_hits;   /* CG solves that stopped at their cap */
    int32_t refinements;     /* mixed mode: outer refinement steps */
    double reaction_norm;    /* ||reaction history|| (solver.h:64) */
    double residual_norm;    /* final Newton residual norm */
    double seconds;          /* device time of the call */
    int32_t direct_solves;   /* linear solves done by the band Cholesky (lpmgpu_desc.direct) */
} lpmgpu_stats;

typedef struct
{
    int32_t n, dim;
    int64_t nbonds;       /* directed bonds */
    int64_t nnzb;         /* full symmetric block count (sum of nconn) */
    int64_t nnz_upper;    /* reference K_pointer[n] */
    int32_t max_bonds;    /* largest bond list */
    int32_t max_conns;    /* largest connection list */
    int64_t device_bytes; /* device memory held by the handle */
} lpmgpu_sizes;

const char *lpmgpu_version(void);
const char *lpmgpu_status_string(int32_t status);
/* message of the last CUDA error seen by this thread (empty when none) */
const char *lpmgpu_last_error(void);

/* Host-side lattice generators, the reference's createPlateSQ2D / createPlateHEX2D /
 * createCuboidSC3D / createCuboidFCC3D (include/utilities.h:93-310) and a BCC generator the
 * reference lacks.  Writes min(count, cap) points to out (3 doubles each); *count gets the total. */
int32_t lpmgpu_generate_lattice(int32_t lattice, double radius, const double box[6], int32_t euler_flag,
                                const double angles[3], double *out, int64_t cap, int64_t *count);

/* Builds the device state: bonds and connections (Assembly ctor, assembly.h:98-106, 213-266),
 * the block pattern, material constants (setParticleProperty), then updateGeometry +
 * updateForceState as the examples do before constructing the solver. */
int32_t lpmgpu_create(const lpmgpu_desc *desc, lpmgpu_solver **out);
int32_t lpmgpu_destroy(lpmgpu_solver *h);
int32_t lpmgpu_get_sizes(const lpmgpu_solver *h, lpmgpu_sizes *out);
/* nb0/nb1/nconn/nlq: n each; bond_p2: nbonds (per particle, layer-0 list then layer-1 list,
 * ascending partner id); conns: nnzb (per particle, ascending id).  Any pointer may be NULL. */
int32_t lpmgpu_get_topology(const lpmgpu_solver *h, int32_t *nb0, int32_t *nb1, int32_t *bond_p2,
                            int32_t *nconn, int32_t *nlq, int32_t *conns);

/* The nonlocal neighbour lists the problem holds (Particle::neighbors_nonlocal, particle.h:37,
 * as Assembly::searchNonlocalNeighbors builds them, assembly.h:118-130: ascending id).  count
 * (n) and ids (the lists concatenated) may be NULL; *total gets the number of ids, 0 when the
 * problem has no lists. */
int32_t lpmgpu_get_nonlocal(const lpmgpu_solver *h, int32_t *count, int32_t *ids, int64_t *total);
/* Assembly::updateGeometry + updateForceState (assembly.h:133-138, 179-191) */
int32_t lpmgpu_update_force_state(lpmgpu_solver *h);
/* Assembly::updateStateVar (assembly.h:162-166): the J2 return map, the elastic-damage or the
 * fatigue particles' energy update */
int32_t lpmgpu_update_state_var(lpmgpu_solver *h);
/* Solver::updateRR (solver.h:112-126); *norm gets ||residual|| */
int32_t lpmgpu_update_rr(lpmgpu_solver *h, double *norm);
/* Stiffness::reset + calcStiffness2D/3D (+ updateStiffnessDispBC when apply_bc) */
int32_t lpmgpu_assemble(lpmgpu_solver *h, int32_t apply_bc);
/* The assembled matrix in the reference's layout: 1-based upper CSR K_pointer[n+1],
 * IK[dim*n+1], JK[nnz_upper], K[nnz_upper] (stiffness.h:24-26, 198-361).  Any may be NULL. */
int32_t lpmgpu_export_ref_csr(const lpmgpu_solver *h, int64_t *K_pointer, int64_t *IK, int64_t *JK, double *K);
/* Solver::LPM_CG (solver.h:277-354) on the current K and residual; disp (host, dim*n) may be NULL */
int32_t lpmgpu_solve_linear(lpmgpu_solver *h, double *disp, lpmgpu_stats *stats);
/* updateForceBC + updateDisplacementBC (solver.h:129-188) */
int32_t lpmgpu_apply_load_step(lpmgpu_solver *h, const lpmgpu_load_step *step);
/* SolverStatic::solveProblemStep (solver_static.h:99-152): returns LPMGPU_ERR_NEWTON on failure */
int32_t lpmgpu_solve_problem_step(lpmgpu_solver *h, const lpmgpu_load_step *step, lpmgpu_stats *stats);
/* One load step of SolverStatic::solveProblem (solver_static.h:72-93) with halve-and-retry */
int32_t lpmgpu_solve_load_step(lpmgpu_solver *h, const lpmgpu_load_step *step, lpmgpu_stats *stats);
/* Assembly::storeStateVar / resetStateVar(true) (assembly.h:141-159) */
int32_t lpmgpu_store_state(lpmgpu_solver *h);
int32_t lpmgpu_reset_state(lpmgpu_solver *h);

/* Direct solve of the current K and residual into disp (host, dim*n; may be NULL), whatever
 * desc.direct says: reverse Cuthill-McKee ordering of the particles (once), the BC-eliminated K
 * into a band, a blocked band Cholesky (once per assembled K) and the two substitutions on the
 * device.  The replacement of Solver::LPM_PARDISO (solver.h:191-274), which refactors the
 * matrix at every call.  LPMGPU_ERR_OUT_OF_MEMORY when the band exceeds 32 GiB (wide 3D
 * problems), LPMGPU_ERR_NOT_SPD for a pivot that is not positive. */
int32_t lpmgpu_solve_direct(lpmgpu_solver *h, double *disp, lpmgpu_stats *stats);
/* The ordering the direct solve uses, on any graph in CSR (host only, no device): rank[i] is
 * vertex i's position under reverse Cuthill-McKee, *bandwidth the largest |rank(i) - rank(j)|
 * over the edges. */
int32_t lpmgpu_band_order(int32_t n, const int32_t *start, const int32_t *adj, int32_t *rank, int64_t *bandwidth);

/* SolverFatigue (include/solver_fatigue.h) on the device.  The cycle loop itself
 * (solveProblemCyclic: readLoad, generateLoadCycle, the dN/dt time map) is host logic and stays
 * with the caller; these are the device steps it calls.
 * lpmgpu_fatigue_solve_step: SolverFatigue::solveProblemStep (solver_fatigue.h:278-302), the BCs,
 *   K from the current state, Newton, no damage loop; LPMGPU_ERR_NEWTON when Newton failed.
 * lpmgpu_fatigue_static_step: one load step of SolverFatigue::solveProblemStatic
 *   (solver_fatigue.h:244-275): the fatigue step with halve-and-retry, and updateStateVar +
 *   storeStateVar after every converged (sub)step.
 * lpmgpu_fatigue_update_damage: SolverFatigue::updateFatigueDamage (solver_fatigue.h:76-126): the
 *   nonlocal average of the local rates, then each damageable particle's damage += rate * dNdt
 *   (ParticleFatigueHCF::updateParticleFatigueDamage, particle_fatigue_hcf.h:148-160);
 *   *any_damaged (may be NULL) gets its return value.
 * lpmgpu_fatigue_cycle: SolverFatigue::solveProblemOneCycle (solver_fatigue.h:221-241): each step
 *   (fatigue step + updateStateVar; a step whose Newton failed is carried on from, as in the
 *   reference, and counted in stats->cuts), then updateFatigueDamage(dNdt), storeStateVar,
 *   updateGeometry, updateForceState. */
int32_t lpmgpu_fatigue_solve_step(lpmgpu_solver *h, const lpmgpu_load_step *step, lpmgpu_stats *stats);
int32_t lpmgpu_fatigue_static_step(lpmgpu_solver *h, const lpmgpu_load_step *step, lpmgpu_stats *stats);
int32_t lpmgpu_fatigue_update_damage(lpmgpu_solver *h, double dNdt, int32_t *any_damaged);
int32_t lpmgpu_fatigue_cycle(lpmgpu_solver *h, const lpmgpu_load_step *steps, int32_t nsteps, double dNdt,
                             lpmgpu_stats *stats, int32_t *any_damaged);

/* Autotuner of the CG launch shape (no counterpart in the reference; the reference's MKL CG has no
 * launch shape).  lpmgpu_autotune re-assembles K from the current state (call it between load
 * steps, after the first, so that the displacement BCs make K definite), then times `iterations` CG iterations of this problem's matrix (the FP32 inner solve in
 * mixed precision) for each candidate grid size: the default (one block per SM, at most one per
 * slice) and 3/4, 1/2, 1/4, 1/8, 1/16 of it.  The fastest stays in force for this handle's later
 * solves; results then differ from the default grid's only by the rounding of the reductions.
 * lpmgpu_set_cg_grid sets the grid directly (0 = the default; values above the default are
 * clamped to it). */
#define LPMGPU_TUNE_MAX 8
typedef struct
{
    int32_t precision;                    /* the precision that was tuned */
    int32_t grid_default, grid_chosen;    /* blocks per CG launch */
    int32_t ncandidates;
    int32_t grid[LPMGPU_TUNE_MAX];        /* candidates, in the order tried */
    double us_per_iter[LPMGPU_TUNE_MAX];  /* their time per CG iteration, microseconds */
} lpmgpu_tune_result;
int32_t lpmgpu_autotune(lpmgpu_solver *h, int32_t iterations, lpmgpu_tune_result *out);
int32_t lpmgpu_set_cg_grid(lpmgpu_solver *h, int32_t grid);
/* Time limit of each grid-barrier wait inside this handle's CG kernel (default 4 s; ns <= 0
 * restores it).  A wait that exceeds it makes every block of the launch return and the solve
 * report LPMGPU_ERR_TIMEOUT; the handle stays usable.  Its use is testing that path: a limit
 * below the natural barrier wait makes the next solve time out.  No counterpart in the reference,
 * whose CG (MKL dcg, solver.h:303-344) has no device waits. */
int32_t lpmgpu_set_wait_limit_ns(lpmgpu_solver *h, int64_t ns);
/* Which stiffness kernel this handle's assemblies use.  0 (the default): the fast form, which
 * sums the reference's terms (Stiffness::calcStiffness2D/3D over localStiffnessANA,
 * stiffness.h:198-361, derivative.h:8-239) in closed form over precomputed 2-hop path lists, with
 * FMA; K agrees with the reference within rounding (about 1e-15 of max|K|).  1: the bit-exact
 * kernel, which reproduces the reference's operator order entry by entry.  The environment
 * variable LPMGPU_ASSEMBLY_EXACT, set when a handle is created, skips building the path lists
 * (the handle then always uses the bit-exact kernel). */
int32_t lpmgpu_set_assembly_exact(lpmgpu_solver *h, int32_t exact);

/* Device state back to host (any pointer may be NULL): xyz n*3, Pin n*3, stress n*6 (s11 s22
 * s33 s23 s13 s12), damage n, damage_visual n, state_var n*nsv (nsv = 7 for J2, 3 for fatigue
 * HCF, else 1),
 * bdamage nbonds, residual dim*n. */
int32_t lpmgpu_read_state(const lpmgpu_solver *h, double *xyz, double *pin, double *stress, double *damage,
                          double *damage_visual, double *state_var, double *bdamage);
int32_t lpmgpu_read_residual(const lpmgpu_solver *h, double *residual);
int32_t lpmgpu_set_xyz(lpmgpu_solver *h, const double *xyz);
/* Device time of the last call's phases, seconds: [0] force/geometry, [1] assembly,
 * [2] linear solves, [3] other */
int32_t lpmgpu_get_phase_times(const lpmgpu_solver *h, double *t4);

/* ---- Per-step output: Assembly::writeDump (include/assembly.h:310-335), the LAMMPS text dump
 * that SolverStatic::solveProblem appends after every load step (solver_static.h:89).
 * lpmgpu_format_dump appends one step for host arrays: xyz, xyz_initial n*3; stress n*6 (s11 s22
 * s33 s23 s13 s12); damage, damage_visual n; state_var n*nsv (column 0 is written); type n or NULL
 * (all 0); box the Assembly's 6 bounds.  The file is opened "a+" as the reference opens it and
 * the bytes are those of the reference's printf conversions for the same values.  Rows are
 * formatted by `threads` host threads (<= 0: all cores) in contiguous chunks, written in order.
 * Needs no device. */
int32_t lpmgpu_format_dump(const char *path, int32_t step, int32_t n, const int32_t *type, const double box[6],
                           const double *xyz, const double *xyz_initial, const double *stress, const double *damage,
                           const double *damage_visual, const double *state_var, int32_t nsv, int32_t threads);
/* The same for the handle's current state, with the coordinates and types given at lpmgpu_create
 * as xyz_initial and type.  The fields are copied to pinned host buffers on the handle's stream
 * after its pending work.  async = 1: the call returns at once and a writer thread of the handle
 * formats and appends the step while the caller goes on (steps are written in call order; at
 * most two are in flight, and a third call waits for one); errors of such steps are returned by
 * lpmgpu_dump_flush.  async = 0: returns once the step is written.  lpmgpu_destroy flushes. */
int32_t lpmgpu_dump_write(lpmgpu_solver *h, const char *path, int32_t step, const double box[6], int32_t threads,
                          int32_t async);
/* waits until every step queued by lpmgpu_dump_write is written; returns the first error among them */
int32_t lpmgpu_dump_flush(lpmgpu_solver *h);

/* Cumulative counters of the handle since creation. */
typedef struct
{
    int64_t kernel_launches;   /* device kernels this handle launched */
    int64_t cg_launches;       /* persistent CG kernel launches */
    int64_t cg_iters;          /* CG iterations over all launches */
    double cg_kernel_seconds;  /* device time inside the CG kernel launches (CUDA events) */
    double assembly_seconds;   /* device time of stiffness assembly + BC elimination */
    double force_seconds;      /* device time of geometry / force / residual passes */
} lpmgpu_counters;
int32_t lpmgpu_get_counters(const lpmgpu_solver *h, lpmgpu_counters *out);
/* The CUDA stream (cudaStream_t) the handle launches on, for callers that time with events. */
int32_t lpmgpu_get_stream(const lpmgpu_solver *h, void **stream);

/* Allocation-free CG, for callers that cannot allocate device memory: a plugin inside a host
 * program that owns all device memory through its own pool or arena, and latency-bound loops
 * that cannot afford cudaMalloc/cudaFree (which may synchronise the device).  No counterpart in
 * the reference (LPM-CPP solves inside Solver::LPM_CG with MKL and allocates per call).
 * Solves A x = b by the same unpreconditioned CG and stopping rule as lpmgpu_solve_linear
 * (||r||^2 <= rtol*||r0||^2 + atol, x0 = 0, maxit <= 0 means rows*dim).  A is block-CSR on the
 * device: rowptr[nrows+1] and colidx[nnzb] (int32), values[nnzb*dim*dim] row-major blocks; b and
 * x are device vectors of rows*dim doubles; stream is a cudaStream_t (NULL = default stream);
 * *iterations (host, may be NULL) gets the iteration count.  The call allocates nothing: its
 * work vectors and reduction words live in a static device array that every GPU loading the
 * library holds (about 8 MiB), so at most 262144 unknowns are accepted (larger sizes return
 * LPMGPU_ERR_INVALID_ARG).  All calls on a device share that array and it keeps the last call's
 * contents, so calls that overlap on the GPU race.  The first call on a device looks the array
 * up (set-up) and should come before any stream capture begins; a cudaDeviceReset invalidates
 * that look-up.  The call waits for its stream before returning.  Returns LPMGPU_ERR_CG_MAXIT
 * when the cap was reached without meeting the tolerance (NaN input included),
 * LPMGPU_ERR_CG_BREAKDOWN when p.Ap == 0, LPMGPU_ERR_TIMEOUT when a device wait gave up; x then
 * holds the last iterate. */
int32_t lpmgpu_cg_bsr_noalloc(int32_t dim, int32_t nrows, const int32_t *rowptr, const int32_t *colidx,
                              const double *values, const double *b, double *x, double rtol, double atol,
                              int64_t maxit, void *stream, int64_t *iterations);

/* ---- Batches: many independent problems advanced together on one GPU (the batched,
 * served form of SolverStatic::solveProblem).  A member is an lpmgpu_solver handle (not owned
 * by the batch) plus its whole load path, copied at lpmgpu_batch_add.  Each member follows
 * exactly the steps of lpmgpu_solve_load_step, load step by load step (halving included); a
 * round advances every member by one piece of device work and solves all members' pending
 * Newton systems in one persistent CG launch.  Members may be added between rounds; finished
 * members may be removed.  A handle must not be used by other calls while it is a running
 * member.  Up to 4096 running members.  Not thread-safe: one host thread per batch. */
typedef struct lpmgpu_batch lpmgpu_batch;

typedef struct
{
    int32_t state;      /* 0 running, 1 done, 2 failed */
    int32_t status;     /* LPMGPU_OK, or the error that stopped the member */
    int32_t steps_done; /* finished load steps */
    int32_t nsteps;
    lpmgpu_stats total; /* summed over the finished load steps */
    int64_t dof_iters;  /* sum over the member's CG iterations of its unknown count */
    double seconds;     /* wall time from lpmgpu_batch_add to completion (or to now) */
} lpmgpu_member_info;

typedef struct
{
    int64_t rounds, cg_launches, members_done, members_failed;
    int64_t cg_iters, dof_iters; /* over members still held by the batch */
    double seconds;              /* wall time inside lpmgpu_batch_run */
    double cg_kernel_seconds;    /* device time of the batched CG launches */
    int32_t fp32_kernel;         /* the mixed members' CG kernel for launches with at least 8
                                    slices of 32 rows per block: 1, 2 single reduction with 1 or 2 SpMV steps
                                    in flight, 3 single reduction with the matrix streamed into
                                    shared memory by bulk copies, 0 two reductions (the batch's tuner
                                    picks it over its first launches unless LPMGPU_BATCH_SR fixes it) */
    int32_t fp32_kernel_small;   /* the same for smaller launches */
    int32_t fp32_tuning;         /* 1 while the tuner is still trying the kernels */
    int32_t pad;
    int64_t solo_solves;         /* linear solves of solo members (lpmgpu_batch_set_solo_bytes) */
} lpmgpu_batch_stats;

int32_t lpmgpu_batch_create(int32_t device, lpmgpu_batch **out);
int32_t lpmgpu_batch_destroy(lpmgpu_batch *b);
/* adds a problem with its load path (steps[0..nsteps)); *member receives its id */
int32_t lpmgpu_batch_add(lpmgpu_batch *b, lpmgpu_solver *h, const lpmgpu_load_step *steps, int32_t nsteps,
                         int32_t *member);
/* one round; *running receives the number of members not yet finished */
/* A fatigue member (the reference's SolverFatigue runs one specimen; no batch counterpart): the
 * nstatic static_steps run as SolverFatigue::solveProblemStatic's steps (solver_fatigue.h:244-275:
 * halve-and-retry, then updateStateVar + storeStateVar), then ncycles cycles of cycle_len steps
 * each (cycle_steps, cycle by cycle) as solveProblemOneCycle runs them (:221-241), cycle c with
 * dN/dt = dndt[c].  Its Newton systems join the batched CG of every round with the other members.
 * Member results: lpmgpu_batch_member_steps gives one record per step; `cuts` of a cycle step
 * counts a Newton failure that was carried on from. */
int32_t lpmgpu_batch_add_fatigue(lpmgpu_batch *b, lpmgpu_solver *h, const lpmgpu_load_step *static_steps,
                                 int32_t nstatic, const lpmgpu_load_step *cycle_steps, int32_t cycle_len,
                                 int32_t ncycles, const double *dndt, int32_t *member);
int32_t lpmgpu_batch_round(lpmgpu_batch *b, int32_t *running);
/* rounds until every member finished */
int32_t lpmgpu_batch_run(lpmgpu_batch *b);
int32_t lpmgpu_batch_member(const lpmgpu_batch *b, int32_t member, lpmgpu_member_info *info);
/* per-load-step statistics of a member (the lpmgpu_stats of each lpmgpu_solve_load_step) */
int32_t lpmgpu_batch_member_steps(const lpmgpu_batch *b, int32_t member, lpmgpu_stats *steps, int32_t cap,
                                  int32_t *count);
/* forgets a finished member (its handle stays with the caller) */
int32_t lpmgpu_batch_remove(lpmgpu_batch *b, int32_t member);
int32_t lpmgpu_batch_get_stats(const lpmgpu_batch *b, lpmgpu_batch_stats *st);
/* CG iterations one batched launch runs before the solves still unfinished pause (they resume
 * in the next round, so one long solve does not hold the other members); 0 = no limit.
 * Default 512. */
int32_t lpmgpu_batch_set_slice(lpmgpu_batch *b, int64_t iterations);
/* Lanes of the batch: its members are dealt to `lanes` groups (by matrix volume), each with its
 * own batched CG launches on an equal share of the SMs.  Lanes progress independently, so one
 * lane's host decisions and per-member kernels overlap the other lanes' CG kernels, and a short
 * solve waits only for the longest solve of its own lane.  Only while no member is running;
 * the default is 1 (LPMGPU_BATCH_LANES in the environment sets a new batch's count).  No
 * counterpart in the reference. */
int32_t lpmgpu_batch_set_lanes(lpmgpu_batch *b, int32_t lanes);
/* Solo members: a member whose CG streams at least `bytes` of matrix per iteration (block values
 * in its CG precision plus block columns) saturates HBM by itself, so batching it with others
 * gains nothing; its linear solves run alone through the single-problem persistent CG (the path
 * of lpmgpu_solve_linear), one at a time between the batched launches, and the rest of its load
 * path stays in the batch's rounds.  Applies to members added afterwards; 0 = no solo members.
 * Default 192 MB.  No counterpart in the reference. */
int32_t lpmgpu_batch_set_solo_bytes(lpmgpu_batch *b, int64_t bytes);

/* ---- Serving: LPM solves submitted while others run (continuous batching).  A request is a
 * problem description plus its load path (both copied at submit).  An admission thread builds a
 * request's device problem once its estimated device memory fits the HBM budget (requests are
 * admitted in arrival order; one larger than the whole budget runs alone); a worker thread adds
 * it to a running batch between two rounds, so its CG iterations share the batched launches of
 * every solve in flight, and when its last load step is done copies its final positions to the
 * host and frees its device memory.  All functions may be called from any host thread. */
typedef struct lpmgpu_server lpmgpu_server;

typedef struct
{
    int32_t state;        /* 0 queued, 1 running, 2 done, 3 failed */
    int32_t status;       /* LPMGPU_OK, or the error that stopped the request */
    int32_t n;            /* particles */
    int32_t steps_done;   /* finished load steps (known once the request is done) */
    int32_t nsteps;
    lpmgpu_stats total;   /* summed over the finished load steps */
    int64_t dof_iters;    /* sum over CG iterations of the unknown count */
    int64_t device_bytes; /* device memory the problem held */
    double t_submit, t_start, t_done; /* seconds since the server was created (-1: not yet) */
} lpmgpu_request_info;

typedef struct
{
    int64_t submitted, queued, running, done, failed, rounds;
    int64_t bytes_in_use, bytes_budget, peak_bytes;
    int32_t worker_status;              /* last error of the batch rounds, LPMGPU_OK if none */
    int32_t pad;
    double latency_p50, latency_p99;    /* seconds from submit to done, over finished requests */
    double seconds;                     /* since the server was created */
} lpmgpu_server_stats;

/* the device memory the server's admission test expects a problem to take (an upper estimate
 * from the particle count, lattice and precision; the problem's real size is in lpmgpu_sizes) */
int32_t lpmgpu_estimate_bytes(const lpmgpu_desc *d, int64_t *bytes);
int32_t lpmgpu_server_create(int32_t device, int64_t hbm_budget_bytes, lpmgpu_server **out);
/* stops both threads; requests not yet fetched are dropped */
int32_t lpmgpu_server_destroy(lpmgpu_server *s);
int32_t lpmgpu_server_set_slice(lpmgpu_server *s, int64_t iterations);
/* lpmgpu_batch_set_lanes for the server's batch, applied once no request is running */
int32_t lpmgpu_server_set_lanes(lpmgpu_server *s, int32_t lanes);
/* lpmgpu_batch_set_solo_bytes for the server's batch, for requests that join it afterwards */
int32_t lpmgpu_server_set_solo_bytes(lpmgpu_server *s, int64_t bytes);
int32_t lpmgpu_server_submit(lpmgpu_server *s, const lpmgpu_desc *d, const lpmgpu_load_step *steps, int32_t nsteps,
                             int64_t *request_id);
/* A fatigue request: the problem and a SolverFatigue run as lpmgpu_batch_add_fatigue takes it
 * (static steps, then ncycles cycles of cycle_len steps with dN/dt dndt[c]), admitted and batched
 * like any request (no counterpart in the reference). */
int32_t lpmgpu_server_submit_fatigue(lpmgpu_server *s, const lpmgpu_desc *d, const lpmgpu_load_step *static_steps,
                                     int32_t nstatic, const lpmgpu_load_step *cycle_steps, int32_t cycle_len,
                                     int32_t ncycles, const double *dndt, int64_t *id);
int32_t lpmgpu_server_poll(lpmgpu_server *s, int64_t request_id, lpmgpu_request_info *info);
/* blocks until the request is done or failed (LPMGPU_OK) or the timeout passed (LPMGPU_ERR_NOT_READY) */
int32_t lpmgpu_server_wait(lpmgpu_server *s, int64_t request_id, double timeout_s, lpmgpu_request_info *info);
/* copies the final positions (n*3 doubles, cap >= n*3) and forgets the request; a failed request
 * returns its error and is forgotten as well */
int32_t lpmgpu_server_result(lpmgpu_server *s, int64_t request_id, double *xyz, int64_t cap);
int32_t lpmgpu_server_get_stats(lpmgpu_server *s, lpmgpu_server_stats *st);

#ifdef __cplusplus
}
#endif
#endif
