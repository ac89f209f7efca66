/*
 * Test infrastructure (oracle): a driver that runs the LPM-CPP reference's own hot path
 * (headers under <reference>/include, compiled unmodified) on a problem described by a
 * small text spec, and writes its results as raw little-endian binaries.  It is built by
 * oracle/Makefile into oracle/_ref/ and is only ever used as a checker or as the timed
 * CPU baseline, never as part of the product.
 *
 * What it calls, in the order of an example's run() (examples/ex1_isoelasticity_2d_hex.cpp:31-120):
 *   UnitCell, createRMatrix, createPlateHEX2D / createPlateSQ2D / createCuboidSC3D /
 *   createCuboidFCC3D (include/utilities.h), Assembly(xyz, box, cell, ptype)
 *   (include/assembly.h:98-106), setParticleProperty (include/particle_elastic.h:70-108,
 *   include/particle_j2plasticity.h:154-198), LoadStep/DispBC/ForceBC, updateGeometry +
 *   updateForceState, SolverStatic (include/solver_static.h:23-24) and either
 *   SolverStatic::solveProblem (include/solver_static.h:65-96; "loop ref") or the same
 *   step loop around SolverStatic::solveProblemStep without the per-step text dump
 *   ("loop step", include/solver_static.h:72-93 minus line 89).
 *
 * Spec format: one directive per line, '#' starts a comment.
 *   lattice hex2d|sq2d|sc3d|fcc3d      radius R       box x0 x1 y0 y1 z0 z1
 *   euler FLAG A1 A2 A3 (radians)      ptype elastic|j2|elastic_damage
 *   edamage K0 K1 CT_RATIO D_THRES    (ParticleElasticDamage::setParticleProperty,
 *                                       include/particle_elastic_damage.h:183-220)
 *   plane_stress 0|1  E v  mu v  critical_bstrain v  j2 sigmay xi H A
 *   nonlocal_L v  nonlocal_cutoff_ratio v  undamaged_type t  init_state_var 0|1
 *   max_iter n  tol_iter v  cg_maxit_cap n
 *   group NAME AXIS OP VALUE [AXIS OP VALUE]     (AXIS 0..2, OP '<' or '>'; conjunction)
 *   settype NAME TYPE                            (assigned in spec order)
 *   steps N
 *   dispbc NAME FLAG STEP [FROM TO]              (FLAG x|y|z, steps FROM..TO-1)
 *   forcebc NAME FX FY FZ [FROM TO]
 *   dumpK STEP   (write the reference CSR after that load step; may repeat)
 *   loop ref|step|once   out DIR   xyz_file PATH (optional: particle coordinates instead of a generator)
 *   groupfile NAME PATH   (group from raw int32 particle ids)   typefile PATH (raw int32 types)
 *   cg_tol RTOL ATOL      (overrides the squared-norm tolerances the reference sets at
 *                          solver.h:312-313; applied inside the MKL stand-in, test use only)
 *   bondfile PATH         (bond list in the reference's text format "id layer p1 p2": the
 *                          Assembly is then built by Assembly(dumpFile, bondFile, cell, ptype),
 *                          include/assembly.h:84-95, from a dump of the coordinates written
 *                          at full precision; pre-cracks by bond exclusion)
 *   tangent 1             (tangent mode: the step of SolverStatic::solveProblemStep with the
 *                          stiffness re-assembled from the current state before every linear
 *                          solve of Solver::NewtonIteration, and not at the start of a damage
 *                          iteration; "loop step|once" only)
 *   dumpfile PATH         (the SolverStatic dumpFile: with "loop ref" the reference's own
 *                          Assembly::writeDump appends every load step there; default /dev/null)
 *   bondprops PATH        (raw f64: Kn[nb], Tv[nb], bdamage[nb] in bond order, written into
 *                          Bond::Kn / Tv / bdamage and bdamage_last (include/bond.h:25-27) after
 *                          setParticleProperty: a heterogeneous material or initial damage)
 *   ptype fatigue_hcf + hcf A B D D_THRES F_LMT_RATIO
 *                         (ParticleFatigueHCF::setParticleProperty, include/particle_fatigue_hcf.h:163-205)
 *   fatigue TYPE N_INTERVAL TMODE TAU   (SolverFatigue, include/solver_fatigue.h: TYPE uniaxial_disp|
 *                          uniaxial_force|dogbone_disp|ct_force (include/load_step_fatigue.h),
 *                          TMODE linear|exponential).  The load steps then run through
 *                          SolverFatigue::solveProblemStatic one at a time, followed by the cycles of
 *                          SolverFatigue::solveProblemCyclic, with the state written after each
 *                          static step and each cycle (outputs numbered on); cycles.txt holds the
 *                          cycle count N and dNdt after each cycle.
 *   fatigue_groups G0 G1 [G2]   (the pt_groups of solveProblemCyclic)
 *   fatigue_load PATH     (the load spectrum, SolverFatigue::readLoad)
 *   solver cg|pardiso     (the SolverMode of the solver: Solver::LPM_CG or Solver::LPM_PARDISO,
 *                          include/solver.h:191-354; default cg)
 *   solve_threads N       (N > 0: omp_set_num_threads(N) once the Assembly is built, so the
 *                          bond and connection searches use every thread and the solve's own
 *                          OpenMP loops use N; with N = 1 the stiffness scatter, which races
 *                          under OpenMP (include/stiffness.h:261-276), is deterministic.  The
 *                          MKL stand-in sizes its own loops by MKL_NUM_THREADS)
 *   cij C11 C12 C44       (C11 > 0: the (C11, C12, C44) overload of setParticleProperty for elastic
 *                          and elastic-damage particles, include/particle_elastic.h:110-140,
 *                          include/particle_elastic_damage.h:218-250)
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>
#include <map>
#include <chrono>

#include "lpm.h"
#include "particle.h"
#include "assembly.h"
#include "utilities.h"
#include "stiffness.h"
#include "load_step.h"
#include "solver_static.h"
#include "solver_fatigue.h"
#include "load_step_fatigue.h"
#ifdef LPM_USE_GPU
/* the one-line switch of an example's run(): SolverStatic -> SolverStaticGPU and
 * SolverFatigue -> SolverFatigueGPU (lpm-cpp_b200/cpp) */
#include "solver_static_gpu.h"
#include "solver_fatigue_gpu.h"
#define LPM_SOLVER SolverStaticGPU
#define LPM_FATIGUE_SOLVER SolverFatigueGPU
#else
#define LPM_SOLVER SolverStatic
#define LPM_FATIGUE_SOLVER SolverFatigue
#endif

static const int NL = 2;

struct Cond
{
    int axis;
    char op;
    double value;
};

struct GroupSpec
{
    std::string name;
    std::vector<Cond> conds;
};

struct DispSpec
{
    std::string group;
    char flag;
    double step;
    int from, to;
};

struct ForceSpec
{
    std::string group;
    double fx, fy, fz;
    int from, to;
};

struct Spec
{
    std::string lattice = "hex2d";
    double radius = 0.1;
    std::array<double, 6> box{0, 1, 0, 1, 0, 1};
    int euler_flag = 0;
    double angles[3] = {0, 0, 0};
    std::string ptype = "elastic";
    double k0 = 0, k1 = 1, ct_ratio = 10, d_thres = 1;
    int plane_stress = 0;
    double E = 69e3, mu = 0.3, critical_bstrain = 1.0;
    double sigmay = 200, xi = 0, H = 0, A = 0;
    double nonlocal_L = 0, nonlocal_cutoff_ratio = 0;
    int undamaged_type = -1;
    int init_state_var = 0;
    int max_iter = 30;
    double tol_iter = 1e-5;
    long long cg_maxit_cap = 0;
    std::vector<GroupSpec> groups;
    std::vector<std::pair<std::string, int>> settypes;
    int steps = 1;
    std::vector<DispSpec> disp;
    std::vector<ForceSpec> force;
    std::vector<int> dumpK;
    int solve_threads = 0;
    std::string loop = "step";
    std::string out = ".";
    std::string xyz_file;
    std::vector<std::pair<std::string, std::string>> groupfiles;
    std::string typefile;
    std::string bondfile;
    std::string bondprops;
    std::string dumpfile = "/dev/null";
    int tangent = 0;
    double cg_rtol = -1, cg_atol = -1;
    double hcf_A = 0, hcf_B = 0, hcf_d = 0, hcf_thres = 1, hcf_flr = 1.108;
    std::string fatigue_type, fatigue_tmode = "linear", fatigue_load;
    int fatigue_interval = 1;
    double fatigue_tau = 1;
    std::vector<std::string> fatigue_groups;
    std::string solver = "cg";
    double C11 = 0, C12 = 0, C44 = 0;
};

static std::vector<int> read_i32(const std::string &path)
{
    std::vector<int> v;
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f)
    {
        std::fprintf(stderr, "cannot open %s\n", path.c_str());
        std::exit(2);
    }
    int x;
    while (std::fread(&x, sizeof(int), 1, f) == 1)
        v.push_back(x);
    std::fclose(f);
    return v;
}

static Spec parse(const char *path)
{
    Spec s;
    std::ifstream f(path);
    if (!f)
    {
        std::fprintf(stderr, "cannot open spec %s\n", path);
        std::exit(2);
    }
    std::string line;
    while (std::getline(f, line))
    {
        auto h = line.find('#');
        if (h != std::string::npos)
            line = line.substr(0, h);
        std::istringstream is(line);
        std::string k;
        if (!(is >> k))
            continue;
        if (k == "lattice") is >> s.lattice;
        else if (k == "radius") is >> s.radius;
        else if (k == "box") for (int i = 0; i < 6; ++i) is >> s.box[i];
        else if (k == "euler") is >> s.euler_flag >> s.angles[0] >> s.angles[1] >> s.angles[2];
        else if (k == "ptype") is >> s.ptype;
        else if (k == "edamage") is >> s.k0 >> s.k1 >> s.ct_ratio >> s.d_thres;
        else if (k == "plane_stress") is >> s.plane_stress;
        else if (k == "E") is >> s.E;
        else if (k == "mu") is >> s.mu;
        else if (k == "critical_bstrain") is >> s.critical_bstrain;
        else if (k == "j2") is >> s.sigmay >> s.xi >> s.H >> s.A;
        else if (k == "nonlocal_L") is >> s.nonlocal_L;
        else if (k == "nonlocal_cutoff_ratio") is >> s.nonlocal_cutoff_ratio;
        else if (k == "undamaged_type") is >> s.undamaged_type;
        else if (k == "init_state_var") is >> s.init_state_var;
        else if (k == "max_iter") is >> s.max_iter;
        else if (k == "tol_iter") is >> s.tol_iter;
        else if (k == "cg_maxit_cap") is >> s.cg_maxit_cap;
        else if (k == "group")
        {
            GroupSpec g;
            is >> g.name;
            Cond c;
            std::string op;
            while (is >> c.axis >> op >> c.value)
            {
                c.op = op[0];
                g.conds.push_back(c);
            }
            s.groups.push_back(g);
        }
        else if (k == "settype")
        {
            std::string n;
            int t;
            is >> n >> t;
            s.settypes.push_back({n, t});
        }
        else if (k == "steps") is >> s.steps;
        else if (k == "dispbc")
        {
            DispSpec d;
            std::string fl;
            is >> d.group >> fl >> d.step;
            d.flag = fl[0];
            d.from = 0;
            d.to = 1 << 30;
            is >> d.from >> d.to;
            s.disp.push_back(d);
        }
        else if (k == "forcebc")
        {
            ForceSpec d;
            is >> d.group >> d.fx >> d.fy >> d.fz;
            d.from = 0;
            d.to = 1 << 30;
            is >> d.from >> d.to;
            s.force.push_back(d);
        }
        else if (k == "solve_threads")
            is >> s.solve_threads;
        else if (k == "dumpK")
        {
            int st;
            is >> st;
            s.dumpK.push_back(st);
        }
        else if (k == "loop") is >> s.loop;
        else if (k == "out") is >> s.out;
        else if (k == "xyz_file") is >> s.xyz_file;
        else if (k == "groupfile")
        {
            std::string n, pth;
            is >> n >> pth;
            s.groupfiles.push_back({n, pth});
        }
        else if (k == "typefile") is >> s.typefile;
        else if (k == "cg_tol") is >> s.cg_rtol >> s.cg_atol;
        else if (k == "bondfile") is >> s.bondfile;
        else if (k == "bondprops") is >> s.bondprops;
        else if (k == "dumpfile") is >> s.dumpfile;
        else if (k == "tangent") is >> s.tangent;
        else if (k == "hcf") is >> s.hcf_A >> s.hcf_B >> s.hcf_d >> s.hcf_thres >> s.hcf_flr;
        else if (k == "fatigue") is >> s.fatigue_type >> s.fatigue_interval >> s.fatigue_tmode >> s.fatigue_tau;
        else if (k == "fatigue_load") is >> s.fatigue_load;
        else if (k == "solver") is >> s.solver;
        else if (k == "cij") is >> s.C11 >> s.C12 >> s.C44;
        else if (k == "fatigue_groups")
        {
            std::string g;
            while (is >> g)
                s.fatigue_groups.push_back(g);
        }
        else
        {
            std::fprintf(stderr, "unknown spec directive '%s'\n", k.c_str());
            std::exit(2);
        }
    }
    return s;
}

template <typename T>
static void write_bin(const std::string &path, const T *data, size_t count)
{
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f)
    {
        std::fprintf(stderr, "cannot write %s\n", path.c_str());
        std::exit(3);
    }
    if (count)
        std::fwrite(data, sizeof(T), count, f);
    std::fclose(f);
}

static double wall()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

static LatticeType lattice_of(const std::string &s)
{
    if (s == "hex2d") return LatticeType::Hexagon2D;
    if (s == "sq2d") return LatticeType::Square2D;
    if (s == "sc3d") return LatticeType::SimpleCubic3D;
    if (s == "fcc3d") return LatticeType::FCC3D;
    if (s == "bcc3d") return LatticeType::BCC3D_1Slip;
    std::fprintf(stderr, "unknown lattice %s\n", s.c_str());
    std::exit(2);
}

/* Assembly(xyz, box, cell, ptype) (assembly.h:98-106), or with a bond file the reference's
 * file constructor: readDump (assembly.h:338-388) of a dump holding the same coordinates, then
 * readBond (assembly.h:391-424). */
static Assembly<NL> make_assembly(std::vector<std::array<double, NDIM>> &xyz, std::array<double, 2 * NDIM> &box,
                                  UnitCell &cell, ParticleType pt, const Spec &sp)
{
    if (sp.bondfile.empty())
        return Assembly<NL>{xyz, box, cell, pt};
    const std::string dump = sp.out + "/assembly_in.dump";
    FILE *f = std::fopen(dump.c_str(), "w");
    if (!f)
    {
        std::fprintf(stderr, "cannot write %s\n", dump.c_str());
        std::exit(3);
    }
    std::fprintf(f, "ITEM: TIMESTEP\n0\nITEM: NUMBER OF ATOMS\n%zu\nITEM: BOX BOUNDS pp pp pp\n", xyz.size());
    for (int k = 0; k < 3; ++k)
        std::fprintf(f, "%.17g %.17g\n", box[2 * k], box[2 * k + 1]);
    std::fprintf(f, "ITEM: ATOMS id type x y z\n");
    for (size_t i = 0; i < xyz.size(); ++i)
        std::fprintf(f, "%zu 0 %.17g %.17g %.17g\n", i, xyz[i][0], xyz[i][1], xyz[i][2]);
    std::fclose(f);
    return Assembly<NL>{dump, sp.bondfile, cell, pt};
}

/* the particle and bond state after a load step or cycle, as raw binaries tagged by its index */
static void write_state(Assembly<NL> &ass, const Spec &sp, const char *tag, int N)
{
    std::vector<double> x(3 * (size_t)N), pin(3 * (size_t)N), stress(6 * (size_t)N), dmg(N), dmgv(N), sv,
        bdmg, dlp;
    int nsv = (int)ass.pt_sys[0]->state_var.size();
    sv.resize((size_t)nsv * N);
    for (Particle<NL> *p : ass.pt_sys)
    {
        for (int k = 0; k < 3; ++k)
        {
            x[3 * p->id + k] = p->xyz[k];
            pin[3 * p->id + k] = p->Pin[k];
        }
        for (int k = 0; k < 6; ++k)
            stress[6 * p->id + k] = p->stress[k];
        dmg[p->id] = p->damage;
        dmgv[p->id] = p->damage_visual;
        for (int k = 0; k < nsv; ++k)
            sv[(size_t)nsv * p->id + k] = p->state_var[k];
    }
    for (Particle<NL> *p : ass.pt_sys)
        for (int l = 0; l < NL; ++l)
            for (Bond<NL> *b : p->bond_layers[l])
            {
                bdmg.push_back(b->bdamage);
                dlp.push_back(b->dLp);
            }
    write_bin(sp.out + "/xyz_" + tag + ".f64", x.data(), x.size());
    write_bin(sp.out + "/pin_" + tag + ".f64", pin.data(), pin.size());
    write_bin(sp.out + "/stress_" + tag + ".f64", stress.data(), stress.size());
    write_bin(sp.out + "/damage_" + tag + ".f64", dmg.data(), dmg.size());
    write_bin(sp.out + "/damage_visual_" + tag + ".f64", dmgv.data(), dmgv.size());
    write_bin(sp.out + "/state_var_" + tag + ".f64", sv.data(), sv.size());
    write_bin(sp.out + "/bdamage_" + tag + ".f64", bdmg.data(), bdmg.size());
    write_bin(sp.out + "/dlp_" + tag + ".f64", dlp.data(), dlp.size());
}

#ifndef LPM_USE_GPU
/* Tangent mode: SolverStatic::solveProblemStep (include/solver_static.h:99-152) whose Newton loop
 * (Solver::NewtonIteration, include/solver.h:55-90) re-assembles the stiffness from the current
 * state (Stiffness::reset + calcStiffness2D/3D + updateStiffnessDispBC, include/stiffness.h)
 * before every solveLinearSystem, instead of once per damage iteration.  Every call is the
 * reference's own code; only the place of the assembly differs. */
static bool tangent_step(SolverStatic<NL> &solv, LoadStep<NL> &load_step)
{
    solv.updateForceBC(load_step);
    solv.updateDisplacementBC(load_step);
    auto &pts = solv.ass.pt_sys;
    int n_newton = 0;
    bool new_damaged = false;
    do
    {
        solv.ass.updateGeometry();
        solv.ass.updateForceState();
        solv.updateRR();
        double norm_residual = cblas_dnrm2(solv.problem_size, solv.stiffness.residual, 1);
        const double norm_reaction =
            cblas_dnrm2((MKL_INT)solv.reaction_force.size(), solv.reaction_force.data(), 1);
        const double tol_multiplier = std::max(norm_residual, norm_reaction);
        int ni = 0;
        while (norm_residual > solv.tol_NR_iter * tol_multiplier)
        {
            if (++ni > solv.max_NR_iter)
            {
                ni = solv.max_NR_iter;
                break;
            }
            solv.stiffness.reset(pts);
            if (pts[0]->cell.dim == 2)
                solv.stiffness.calcStiffness2D(pts);
            else
                solv.stiffness.calcStiffness3D(pts);
            solv.stiffness.updateStiffnessDispBC(pts);
            solv.solveLinearSystem();
            solv.ass.updateGeometry();
            solv.ass.updateForceState();
            solv.updateRR();
            norm_residual = cblas_dnrm2(solv.problem_size, solv.stiffness.residual, 1);
        }
        n_newton = ni;
        if (n_newton >= solv.max_NR_iter)
            break;
        solv.ass.updateStateVar();
        new_damaged = solv.updateStaticDamage();
        solv.ass.storeStateVar();
        if (new_damaged)
        {
            solv.ass.updateGeometry();
            solv.ass.updateForceState();
        }
    } while (new_damaged);
    return n_newton < solv.max_NR_iter;
}
#endif

#ifdef LPM_USE_GPU
/* the device solver counts its own linear solves and CG iterations */
#define DEVICE_COUNTS_BEGIN const long long gn0 = solv.totals.newton_solves, gc0 = solv.totals.cg_iters;
#define DEVICE_COUNTS_END                                                                                             \
    st1.cg_solves = st0.cg_solves + (solv.totals.newton_solves - gn0);                                                 \
    st1.cg_iterations = st0.cg_iterations + (solv.totals.cg_iters - gc0);
#else
#define DEVICE_COUNTS_BEGIN
#define DEVICE_COUNTS_END
#endif

static FatigueLoadType fatigue_type_of(const std::string &s)
{
    if (s == "uniaxial_disp") return FatigueLoadType::LoadUniaxialDisp;
    if (s == "uniaxial_force") return FatigueLoadType::LoadUniaxialForce;
    if (s == "dogbone_disp") return FatigueLoadType::LoadDogBoneDisp;
    if (s == "ct_force") return FatigueLoadType::LoadCTForce;
    std::fprintf(stderr, "unknown fatigue load type %s\n", s.c_str());
    std::exit(2);
}

static void log_line(FILE *log, int s, const lpm_shim_stats &st0, const lpm_shim_stats &st1, double wall_s, int cuts,
                     double rn)
{
    std::fprintf(log, "%d %lld %lld %.6f %.6f %.6f %.6f %d %.17g %lld\n", s, st1.cg_solves - st0.cg_solves,
                 st1.cg_iterations - st0.cg_iterations, wall_s, st1.spmv_seconds - st0.spmv_seconds,
                 st1.cg_seconds - st0.cg_seconds, st1.create_seconds - st0.create_seconds, cuts, rn,
                 st1.cg_failures - st0.cg_failures);
    std::fflush(log);
}

/* SolverFatigue (include/solver_fatigue.h): the spec's load steps through solveProblemStatic one at
 * a time, then the cycles of solveProblemCyclic.  The cycle loop is the reference's
 * (solver_fatigue.h:183-218: generateLoadCycle, the dN/dt time map, solveProblemOneCycle,
 * N += (int)dNdt while N < n_cycles) with the state written after each cycle in place of its
 * printout and dump. */
static int run_fatigue(Assembly<NL> &ass, std::map<std::string, std::vector<Particle<NL> *>> &groups,
                       std::vector<LoadStep<NL>> &load, const Spec &sp, int N, int dim, double setup_s)
{
    const TimeMapMode tm = (sp.fatigue_tmode == "exponential") ? TimeMapMode::Exponential : TimeMapMode::Linear;
    const SolverMode sm = (sp.solver == "pardiso") ? SolverMode::PARDISO : SolverMode::CG;
    LPM_FATIGUE_SOLVER<NL> solv{sp.undamaged_type, ass, StiffnessMode::Analytical, sm, tm, sp.fatigue_tau,
                                sp.dumpfile, sp.max_iter, sp.tol_iter};
#ifdef LPM_USE_GPU
    if (sp.cg_rtol >= 0 || sp.cg_atol >= 0)
        solv.setCGTolerance(sp.cg_rtol >= 0 ? sp.cg_rtol : 1e-12, sp.cg_atol >= 0 ? sp.cg_atol : 1e-12);
#endif
    FILE *log = std::fopen((sp.out + "/steps.txt").c_str(), "w");
    std::fprintf(log, "# N %d dim %d setup_s %.6f threads %d\n", N, dim, setup_s, omp_get_max_threads());
    std::fprintf(log, "# step newton_solves cg_iters wall_s spmv_s cg_s create_s cuts reaction_norm cg_fail\n");
    int start_index = 0, idx = 0;
    char tag[32];
    for (int s = 0; s < sp.steps; ++s, ++idx)
    {
        lpm_shim_stats st0 = lpm_shim_stats_g;
        DEVICE_COUNTS_BEGIN
        const double t0 = wall();
        std::vector<LoadStep<NL>> one{load[s]};
        solv.solveProblemStatic(one, start_index);
        lpm_shim_stats st1 = lpm_shim_stats_g;
        DEVICE_COUNTS_END
        log_line(log, idx, st0, st1, wall() - t0, (int)one.size() - 1,
                 cblas_dnrm2((MKL_INT)solv.reaction_force.size(), solv.reaction_force.data(), 1));
        std::snprintf(tag, sizeof tag, "%03d", idx);
        write_state(ass, sp, tag, N);
    }
    if (!sp.fatigue_load.empty())
    {
        const FatigueLoadType lt = fatigue_type_of(sp.fatigue_type);
        std::vector<std::vector<Particle<NL> *>> pg;
        for (const std::string &g : sp.fatigue_groups)
            pg.push_back(groups[g]);
        solv.readLoad(sp.fatigue_load);
        FILE *cyc = std::fopen((sp.out + "/cycles.txt").c_str(), "w");
        const double n_cycles = 0.5 * (solv.load_spectrum.size() - 1);
        double t = 0, dNdt = 1;
        int Nc = 0;
        do
        {
            lpm_shim_stats st0 = lpm_shim_stats_g;
            DEVICE_COUNTS_BEGIN
            const double t0 = wall();
            std::vector<LoadStep<NL>> load_cycle = solv.generateLoadCycle(lt, Nc, sp.fatigue_interval, pg);
            dNdt = (tm == TimeMapMode::Linear) ? func_dNdt_linear(sp.fatigue_tau) : func_dNdt_exponental(sp.fatigue_tau, t++);
            solv.solveProblemOneCycle(load_cycle, dNdt);
            Nc += (int)dNdt;
            lpm_shim_stats st1 = lpm_shim_stats_g;
            DEVICE_COUNTS_END
            log_line(log, idx, st0, st1, wall() - t0, 0,
                     cblas_dnrm2((MKL_INT)solv.reaction_force.size(), solv.reaction_force.data(), 1));
            std::fprintf(cyc, "%d %.17g\n", Nc, dNdt);
            std::snprintf(tag, sizeof tag, "%03d", idx++);
            write_state(ass, sp, tag, N);
        } while (Nc < n_cycles);
        std::fclose(cyc);
    }
    std::fclose(log);
    return 0;
}

int main(int argc, char **argv)
{
    if (argc < 2)
    {
        std::fprintf(stderr, "usage: lpm_ref SPEC\n");
        return 2;
    }
    Spec sp = parse(argv[1]);
    if (sp.tangent && sp.loop == "ref")
    {
        std::fprintf(stderr, "tangent mode needs loop step or once\n");
        return 2;
    }
    lpm_shim_stats_g.cg_maxit_override = sp.cg_maxit_cap;
    lpm_shim_stats_g.cg_rtol_override = sp.cg_rtol;
    lpm_shim_stats_g.cg_atol_override = sp.cg_atol;
    const double t_setup0 = wall();

    UnitCell cell(lattice_of(sp.lattice), sp.radius);
    double *R = createRMatrix(sp.euler_flag, sp.angles);
    std::array<double, 2 * NDIM> box = sp.box;
    std::vector<std::array<double, NDIM>> xyz;
    if (!sp.xyz_file.empty())
    {
        FILE *f = std::fopen(sp.xyz_file.c_str(), "rb");
        if (!f)
        {
            std::fprintf(stderr, "cannot open %s\n", sp.xyz_file.c_str());
            return 2;
        }
        std::array<double, NDIM> p;
        while (std::fread(p.data(), sizeof(double), 3, f) == 3)
            xyz.push_back(p);
        std::fclose(f);
    }
    else if (sp.lattice == "hex2d") xyz = createPlateHEX2D(box, cell, R);
    else if (sp.lattice == "sq2d") xyz = createPlateSQ2D(box, cell, R);
    else if (sp.lattice == "sc3d") xyz = createCuboidSC3D(box, cell, R);
    else if (sp.lattice == "fcc3d") xyz = createCuboidFCC3D(box, cell, R);
    else
    {
        std::fprintf(stderr, "lattice %s needs xyz_file\n", sp.lattice.c_str());
        return 2;
    }

    ParticleType pt = (sp.ptype == "j2")               ? ParticleType::J2Plasticity
                      : (sp.ptype == "elastic_damage") ? ParticleType::ElasticDamage
                      : (sp.ptype == "fatigue_hcf")    ? ParticleType::FatigueHCF
                                                       : ParticleType::Elastic;
    Assembly<NL> ass = make_assembly(xyz, box, cell, pt, sp);
    const int N = ass.nparticle;
    const int dim = cell.dim;

    std::map<std::string, std::vector<Particle<NL> *>> groups;
    for (auto &g : sp.groups)
    {
        std::vector<Particle<NL> *> mem;
        for (Particle<NL> *p : ass.pt_sys)
        {
            bool ok = true;
            for (auto &c : g.conds)
                ok = ok && ((c.op == '<') ? (p->xyz[c.axis] < c.value) : (p->xyz[c.axis] > c.value));
            if (ok)
                mem.push_back(p);
        }
        groups[g.name] = mem;
    }
    for (auto &gf : sp.groupfiles)
    {
        std::vector<Particle<NL> *> mem;
        for (int id : read_i32(gf.second))
            mem.push_back(ass.pt_sys[id]);
        groups[gf.first] = mem;
    }
    if (!sp.typefile.empty())
    {
        std::vector<int> t = read_i32(sp.typefile);
        for (Particle<NL> *p : ass.pt_sys)
            p->type = t[p->id];
    }
    for (auto &st : sp.settypes)
        for (Particle<NL> *p : groups[st.first])
            p->type = st.second;

    for (Particle<NL> *p : ass.pt_sys)
    {
        if (pt == ParticleType::J2Plasticity)
            dynamic_cast<ParticleJ2Plasticity<NL> *>(p)->setParticleProperty(
                sp.nonlocal_L, sp.plane_stress != 0, sp.E, sp.mu, sp.sigmay, sp.xi, sp.H, sp.A, sp.critical_bstrain);
        else if (pt == ParticleType::ElasticDamage && sp.C11 > 0)
            dynamic_cast<ParticleElasticDamage<NL> *>(p)->setParticleProperty(sp.nonlocal_L, sp.C11, sp.C12, sp.C44,
                                                                              sp.k0, sp.k1, sp.ct_ratio, sp.d_thres);
        else if (pt == ParticleType::ElasticDamage)
            dynamic_cast<ParticleElasticDamage<NL> *>(p)->setParticleProperty(
                sp.nonlocal_L, sp.plane_stress != 0, sp.E, sp.mu, sp.k0, sp.k1, sp.ct_ratio, sp.d_thres);
        else if (pt == ParticleType::FatigueHCF)
            dynamic_cast<ParticleFatigueHCF<NL> *>(p)->setParticleProperty(
                sp.nonlocal_L, sp.plane_stress != 0, sp.E, sp.mu, sp.hcf_A, sp.hcf_B, sp.hcf_d, sp.hcf_thres, sp.hcf_flr);
        else if (sp.C11 > 0)
            dynamic_cast<ParticleElastic<NL> *>(p)->setParticleProperty(sp.nonlocal_L, sp.C11, sp.C12, sp.C44,
                                                                        sp.critical_bstrain);
        else
            dynamic_cast<ParticleElastic<NL> *>(p)->setParticleProperty(sp.nonlocal_L, sp.plane_stress != 0, sp.E,
                                                                        sp.mu, sp.critical_bstrain);
    }

    if (!sp.bondprops.empty())
    {
        std::vector<double> v;
        FILE *f = std::fopen(sp.bondprops.c_str(), "rb");
        if (!f)
        {
            std::fprintf(stderr, "cannot open %s\n", sp.bondprops.c_str());
            return 2;
        }
        double x;
        while (std::fread(&x, sizeof(double), 1, f) == 1)
            v.push_back(x);
        std::fclose(f);
        size_t nb = 0;
        for (Particle<NL> *p : ass.pt_sys)
            for (int l = 0; l < NL; ++l)
                nb += p->bond_layers[l].size();
        if (v.size() != 3 * nb)
        {
            std::fprintf(stderr, "bondprops holds %zu values, expected 3 x %zu bonds\n", v.size(), nb);
            return 2;
        }
        size_t k = 0;
        for (Particle<NL> *p : ass.pt_sys)
            for (int l = 0; l < NL; ++l)
                for (Bond<NL> *b : p->bond_layers[l])
                {
                    b->Kn = v[k];
                    b->Tv = v[nb + k];
                    b->bdamage = b->bdamage_last = v[2 * nb + k];
                    ++k;
                }
    }

    std::vector<LoadStep<NL>> load;
    for (int s = 0; s < sp.steps; ++s)
    {
        LoadStep<NL> step;
        for (auto &d : sp.disp)
            if (s >= d.from && s < d.to)
                step.dispBCs.push_back(DispBC<NL>(groups[d.group], LoadMode::Relative, d.flag, d.step));
        for (auto &f : sp.force)
            if (s >= f.from && s < f.to)
                step.forceBCs.push_back(ForceBC<NL>(groups[f.group], LoadMode::Relative, f.fx, f.fy, f.fz));
        load.push_back(step);
    }

    if (sp.nonlocal_cutoff_ratio > 0)
        ass.searchNonlocalNeighbors(sp.nonlocal_cutoff_ratio);
    ass.updateGeometry();
    ass.updateForceState();
    if (sp.init_state_var)
        ass.updateStateVar();

    const SolverMode sm = (sp.solver == "pardiso") ? SolverMode::PARDISO : SolverMode::CG;
    LPM_SOLVER<NL> solv{sp.undamaged_type, ass, StiffnessMode::Analytical, sm, sp.dumpfile,
                        sp.max_iter, sp.tol_iter};
#ifdef LPM_USE_GPU
    if (sp.cg_rtol >= 0 || sp.cg_atol >= 0)
        solv.setCGTolerance(sp.cg_rtol >= 0 ? sp.cg_rtol : 1e-12, sp.cg_atol >= 0 ? sp.cg_atol : 1e-12);
#endif
    if (sp.solve_threads > 0)
        omp_set_num_threads(sp.solve_threads);
    const double t_setup1 = wall();

    /* setup outputs: coordinates, bonds (per particle: layer-0 list then layer-1 list), conns */
    {
        std::vector<double> x0(3 * (size_t)N);
        std::vector<int> nb0(N), nb1(N), bp2, nconn(N), nlq(N), conns;
        for (Particle<NL> *p : ass.pt_sys)
        {
            for (int k = 0; k < 3; ++k)
                x0[3 * p->id + k] = p->xyz_initial[k];
            nb0[p->id] = (int)p->bond_layers[0].size();
            nb1[p->id] = (int)p->bond_layers[1].size();
            nconn[p->id] = p->nconn;
            nlq[p->id] = p->nconn_largeq;
        }
        for (Particle<NL> *p : ass.pt_sys)
        {
            for (int l = 0; l < NL; ++l)
                for (Bond<NL> *b : p->bond_layers[l])
                    bp2.push_back(b->p2->id);
            for (Particle<NL> *c : p->conns)
                conns.push_back(c->id);
        }
        std::vector<int> types(N);
        for (Particle<NL> *p : ass.pt_sys)
            types[p->id] = p->type;
        write_bin(sp.out + "/xyz0.f64", x0.data(), x0.size());
        write_bin(sp.out + "/nb0.i32", nb0.data(), nb0.size());
        write_bin(sp.out + "/nb1.i32", nb1.data(), nb1.size());
        write_bin(sp.out + "/bond_p2.i32", bp2.data(), bp2.size());
        write_bin(sp.out + "/nconn.i32", nconn.data(), nconn.size());
        write_bin(sp.out + "/nlq.i32", nlq.data(), nlq.size());
        write_bin(sp.out + "/conns.i32", conns.data(), conns.size());
        write_bin(sp.out + "/type.i32", types.data(), types.size());
        std::vector<double> pin0(3 * (size_t)N);
        for (Particle<NL> *p : ass.pt_sys)
            for (int k = 0; k < 3; ++k)
                pin0[3 * p->id + k] = p->Pin[k];
        write_bin(sp.out + "/pin_init.f64", pin0.data(), pin0.size());
    }

    if (!sp.fatigue_type.empty())
        return run_fatigue(ass, groups, load, sp, N, dim, t_setup1 - t_setup0);
    FILE *log = std::fopen((sp.out + "/steps.txt").c_str(), "w");
    std::fprintf(log, "# N %d dim %d setup_s %.6f threads %d\n", N, dim, t_setup1 - t_setup0, omp_get_max_threads());
    std::fprintf(log, "# step newton_solves cg_iters wall_s spmv_s cg_s create_s cuts reaction_norm cg_fail\n");

    int start_index = 0;
    for (int s = 0; s < sp.steps; ++s)
    {
        lpm_shim_stats st0 = lpm_shim_stats_g;
#ifdef LPM_USE_GPU
        const long long gpu_newton0 = solv.totals.newton_solves, gpu_cg0 = solv.totals.cg_iters;
#endif
        double t0 = wall();
        int cuts = 0;
        if (sp.loop == "once")
        {
            /* one SolverStatic::solveProblemStep call, no retry: a bounded sample of the step */
            double dt = 1;
#ifndef LPM_USE_GPU
            if (sp.tangent)
                cuts = tangent_step(solv, load[s]) ? 0 : -1;
            else
#endif
                cuts = solv.solveProblemStep(load[s], dt) ? 0 : -1;
        }
        else if (sp.loop == "ref")
        {
            std::vector<LoadStep<NL>> one{load[s]};
            solv.solveProblem(one, start_index);
            cuts = (int)one.size() - 1;
        }
        else
        {
            /* the loop of SolverStatic::solveProblem (include/solver_static.h:72-93) without the dump */
            std::vector<LoadStep<NL>> one{load[s]};
            int n_step = (int)one.size();
            double dt = 1;
            for (int i = 0; i < n_step; i++)
            {
#ifndef LPM_USE_GPU
                bool ok = sp.tangent ? tangent_step(solv, one[i]) : solv.solveProblemStep(one[i], dt);
#else
                bool ok = solv.solveProblemStep(one[i], dt);
#endif
                if (!ok)
                {
#ifdef LPM_USE_GPU
                    lpmgpu_reset_state(solv.handle());
#else
                    solv.ass.resetStateVar(true);
#endif
                    one[i].loadCutHalf();
                    one.insert(one.begin() + i, one[i]);
                    ++n_step;
                    ++cuts;
                    --i;
                    if (cuts > 40)
                    {
                        std::fprintf(stderr, "too many load cuts at step %d\n", s);
                        return 4;
                    }
                }
            }
            start_index += n_step;
        }
        double t1 = wall();
        lpm_shim_stats st1 = lpm_shim_stats_g;
#ifdef LPM_USE_GPU
        /* the device solver counts its own linear solves and CG iterations */
        st1.cg_solves = st0.cg_solves + (solv.totals.newton_solves - gpu_newton0);
        st1.cg_iterations = st0.cg_iterations + (solv.totals.cg_iters - gpu_cg0);
#endif
        double rn = cblas_dnrm2((MKL_INT)solv.reaction_force.size(), solv.reaction_force.data(), 1);
        std::fprintf(log, "%d %lld %lld %.6f %.6f %.6f %.6f %d %.17g %lld\n", s, st1.cg_solves - st0.cg_solves,
                     st1.cg_iterations - st0.cg_iterations, t1 - t0, st1.spmv_seconds - st0.spmv_seconds,
                     st1.cg_seconds - st0.cg_seconds, st1.create_seconds - st0.create_seconds, cuts, rn,
                     st1.cg_failures - st0.cg_failures);
        std::fflush(log);

        char tag[32];
        std::snprintf(tag, sizeof tag, "%03d", s);
        write_state(ass, sp, tag, N);

        bool dump = false;
        for (int d : sp.dumpK)
            dump = dump || (d == s);
        if (dump)
        {
            const long long nnz = solv.stiffness.K_pointer[N];
            write_bin(sp.out + "/K_pointer_" + tag + ".i64", solv.stiffness.K_pointer, (size_t)N + 1);
            write_bin(sp.out + "/IK_" + tag + ".i64", solv.stiffness.IK, (size_t)dim * N + 1);
            write_bin(sp.out + "/JK_" + tag + ".i64", solv.stiffness.JK, (size_t)nnz);
            write_bin(sp.out + "/K_" + tag + ".f64", solv.stiffness.K_global, (size_t)nnz);
        }
    }
    std::fclose(log);
    return 0;
}
