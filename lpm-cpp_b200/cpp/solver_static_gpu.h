// SolverStaticGPU<nlayer>: a drop-in for LPM-CPP's SolverStatic<nlayer> (include/solver_static.h:17-29)
// that runs the implicit quasi-static load step on the GPU through liblpmgpu (include/lpmgpu.h).
//
// An example's run() switches with one line, the constructor arguments unchanged:
//
//     SolverStatic<n_layer> solv{undamaged_pt_type, pt_ass, StiffnessMode::Analytical, SolverMode::CG,
//                                dumpFile, max_iter, tol_iter};
//  -> SolverStaticGPU<n_layer> solv{undamaged_pt_type, pt_ass, StiffnessMode::Analytical, SolverMode::CG,
//                                   dumpFile, max_iter, tol_iter};
//
// Include this header after the LPM-CPP headers it works with (lpm.h, assembly.h, load_step.h and
// the particle headers assembly.h includes) and link liblpmgpu.so.  SolverFatigueGPU is in
// solver_fatigue_gpu.h.  The constructor packs the
// Assembly - coordinates, particle types, the bond lists exactly as the Assembly holds them, each
// bond's Kn/Tv and damage, the J2 parameters - and builds the device state.  solveProblem /
// solveProblemStep keep the reference's contract: the same load-step loop with halve-and-retry
// (the load vector and start_index change as in solver_static.h:65-96), a text dump per step
// through Assembly::writeDump, and afterwards `stiffness.K_pointer / IK / JK / K_global` hold the
// last assembled matrix in the reference's layout.  Particle fields (xyz, Pin, stress, damage,
// damage_visual, state_var, bond damage) are written back after every step.
#pragma once

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "lpmgpu.h"

namespace lpmgpu_detail
{
// ParticleElastic keeps critical_bstrain private (include/particle_elastic.h:18).  Its value is
// read through a member pointer formed in an explicit template instantiation, where access
// checking does not apply, so the LPM-CPP headers stay unmodified.
template <class Tag>
struct member_slot
{
    static typename Tag::type ptr;
};
template <class Tag>
typename Tag::type member_slot<Tag>::ptr;

template <class Tag, typename Tag::type P>
struct member_reader : member_slot<Tag>
{
    struct filler
    {
        filler() { member_slot<Tag>::ptr = P; }
    };
    static filler instance;
};
template <class Tag, typename Tag::type P>
typename member_reader<Tag, P>::filler member_reader<Tag, P>::instance;

struct ElasticCriticalStrain
{
    typedef double ParticleElastic<2>::*type;
};
template struct member_reader<ElasticCriticalStrain, &ParticleElastic<2>::critical_bstrain>;

inline int lattice_code(LatticeType t)
{
    switch (t)
    {
    case LatticeType::Square2D: return LPMGPU_SQUARE2D;
    case LatticeType::Hexagon2D: return LPMGPU_HEXAGON2D;
    case LatticeType::SimpleCubic3D: return LPMGPU_SC3D;
    case LatticeType::FCC3D: return LPMGPU_FCC3D;
    default: return LPMGPU_BCC3D;
    }
}

inline void check(int32_t status, const char *what)
{
    if (status != LPMGPU_OK)
        throw std::runtime_error(std::string(what) + ": " + lpmgpu_status_string(status) + " " + lpmgpu_last_error());
}
} // namespace lpmgpu_detail

template <int nlayer>
class SolverStaticGPU
{
public:
    int undamaged_pt_type{0};
    int problem_size{0}, max_NR_iter{0};
    double tol_NR_iter{0};
    std::string dumpFile;
    // The reference keeps every reaction force it ever saw (solver.h:25, 122-123) and uses only
    // its norm; this vector holds that norm as its single element, so cblas_dnrm2 over it gives
    // the same number.
    std::vector<double> reaction_force;
    Assembly<nlayer> ass;
    bool export_stiffness{true}; // materialise `stiffness` after each solveProblem
    lpmgpu_stats totals{};       // Newton solves and CG iterations summed over all calls

    struct StiffnessArrays
    {
        MKL_INT *K_pointer{nullptr}, *IK{nullptr}, *JK{nullptr};
        double *K_global{nullptr};
        std::vector<MKL_INT> kp, ik, jk;
        std::vector<double> kv;
    } stiffness;

    SolverStaticGPU(const int &p_undamaged, Assembly<nlayer> &p_ass, const StiffnessMode &p_stiff_mode,
                    const SolverMode &p_sol_mode, const std::string &p_dumpFile, const int &p_niter,
                    const double &p_tol, int precision = LPMGPU_FP64, int device = 0)
        : undamaged_pt_type{p_undamaged}, max_NR_iter{p_niter}, tol_NR_iter{p_tol}, dumpFile{p_dumpFile},
          ass(p_ass)
    {
        // SolverMode::PARDISO, the direct solve of Solver::LPM_PARDISO (solver.h:191-274): the
        // device CG to a relative residual of 1e-12 (squared-norm test 1e-24) instead of the
        // reference CG's 1e-6, and the device's band Cholesky for a system the CG cannot solve.
        if (p_sol_mode == SolverMode::PARDISO)
        {
            direct_ = 2;
            cg_rtol_ = 1e-24;
            cg_atol_ = 0.0;
        }
        if (p_stiff_mode != StiffnessMode::Analytical)
            throw std::runtime_error("SolverStaticGPU supports StiffnessMode::Analytical only");
        create(precision, device);
    }

    ~SolverStaticGPU()
    {
        if (h_)
            lpmgpu_destroy(h_);
    }

    SolverStaticGPU(const SolverStaticGPU &) = delete;
    SolverStaticGPU &operator=(const SolverStaticGPU &) = delete;

    // Squared-norm CG test ||r||^2 <= rtol ||r0||^2 + atol; the reference fixes 1e-12 / 1e-12.
    void setCGTolerance(double rtol, double atol)
    {
        cg_rtol_ = rtol;
        cg_atol_ = atol;
        rebuild_needed_ = true;
    }

    // SolverStatic::solveProblemStep (solver_static.h:99-152)
    bool solveProblemStep(LoadStep<nlayer> &load_step, double &dt)
    {
        (void)dt;
        ensure_tolerances();
        CStep c(load_step);
        lpmgpu_stats st{};
        const int32_t r = lpmgpu_solve_problem_step(h_, &c.step, &st);
        if (r != LPMGPU_OK && r != LPMGPU_ERR_NEWTON)
            lpmgpu_detail::check(r, "lpmgpu_solve_problem_step");
        totals.newton_solves += st.newton_solves;
        totals.cg_iters += st.cg_iters;
        totals.cg_maxit_hits += st.cg_maxit_hits;
        totals.direct_solves += st.direct_solves;
        reaction_force.assign(1, st.reaction_norm);
        write_back();
        return r == LPMGPU_OK;
    }

    // SolverStatic::solveProblem (solver_static.h:65-96)
    void solveProblem(std::vector<LoadStep<nlayer>> &load, int &start_index)
    {
        int n_step = (int)load.size();
        double dt = 1;
        for (int i = 0; i < n_step; i++)
        {
        restart:
            printf("Loading step-%d, iteration starts:\n", i + start_index);
            const bool is_converged = solveProblemStep(load[i], dt);
            if (!is_converged)
            {
                lpmgpu_detail::check(lpmgpu_reset_state(h_), "lpmgpu_reset_state");
                load[i].loadCutHalf();
                load.insert(load.begin() + i, load[i]);
                ++n_step;
                printf("Step-%d not converging\n\n", i + start_index);
                goto restart;
            }
            if (!dumpFile.empty())
                ass.writeDump(dumpFile, i + start_index);
        }
        start_index += n_step;
        if (export_stiffness)
            export_K();
    }

    lpmgpu_solver *handle() { return h_; }

protected:
    lpmgpu_solver *h_{nullptr};
    int precision_{LPMGPU_FP64}, device_{0};
    double cg_rtol_{1e-12}, cg_atol_{1e-12};
    int direct_{0}; // lpmgpu_desc.direct
    bool rebuild_needed_{false};

    struct CStep
    {
        std::vector<std::vector<int32_t>> ids;
        std::vector<lpmgpu_dispbc> d;
        std::vector<lpmgpu_forcebc> f;
        lpmgpu_load_step step{};

        explicit CStep(LoadStep<nlayer> &s)
        {
            for (auto &bc : s.dispBCs)
            {
                if (bc.load_mode != LoadMode::Relative)
                    throw std::runtime_error("SolverStaticGPU supports LoadMode::Relative only");
                ids.emplace_back();
                for (auto *p : bc.group)
                    ids.back().push_back(p->id);
                const int flag = bc.flag == 'x' ? 0 : (bc.flag == 'y' ? 1 : 2);
                d.push_back({nullptr, (int32_t)ids.back().size(), flag, bc.step});
            }
            for (auto &bc : s.forceBCs)
            {
                if (bc.load_mode != LoadMode::Relative)
                    throw std::runtime_error("SolverStaticGPU supports LoadMode::Relative only");
                ids.emplace_back();
                for (auto *p : bc.group)
                    ids.back().push_back(p->id);
                f.push_back({nullptr, (int32_t)ids.back().size(), bc.fx, bc.fy, bc.fz});
            }
            size_t q = 0;
            for (auto &x : d)
                x.ids = ids[q++].data();
            for (auto &x : f)
                x.ids = ids[q++].data();
            step = {d.data(), (int32_t)d.size(), f.data(), (int32_t)f.size()};
        }
    };

    void create(int precision, int device)
    {
        precision_ = precision;
        device_ = device;
        auto &pts = ass.pt_sys;
        const int n = (int)pts.size();
        const int dim = pts[0]->cell.dim;
        problem_size = dim * n;
        std::vector<double> xyz(3 * (size_t)n), kn, tv, dmg;
        std::vector<int32_t> type(n), nb0(n), nb1(n), p2;
        for (auto *p : pts)
        {
            for (int k = 0; k < 3; ++k)
                xyz[3 * (size_t)p->id + k] = p->xyz[k];
            type[p->id] = p->type;
            nb0[p->id] = (int32_t)p->bond_layers[0].size();
            nb1[p->id] = (int32_t)p->bond_layers[1].size();
        }
        for (auto *p : pts) // pt_sys is in id order (particle.h:68, assembly.h:196)
            for (int l = 0; l < nlayer; ++l)
                for (auto *b : p->bond_layers[l])
                {
                    p2.push_back(b->p2->id);
                    kn.push_back(b->Kn);
                    tv.push_back(b->Tv);
                    dmg.push_back(b->bdamage);
                }
        lpmgpu_desc d{};
        d.lattice = lpmgpu_detail::lattice_code(pts[0]->cell.lattice);
        d.n = n;
        d.xyz = xyz.data();
        d.type = type.data();
        d.radius = pts[0]->cell.radius;
        if (auto *j2 = dynamic_cast<ParticleJ2Plasticity<nlayer> *>(pts[0]))
        {
            d.ptype = LPMGPU_J2;
            d.E = j2->E;
            d.mu = j2->mu;
            d.sigmay = j2->sigmay;
            d.xi = j2->xi;
            d.H = j2->H;
            d.A = j2->A;
            d.critical_bstrain = j2->critical_bstrain;
        }
        else if (auto *el = dynamic_cast<ParticleElastic<nlayer> *>(pts[0]))
        {
            d.ptype = LPMGPU_ELASTIC;
            d.critical_bstrain = el->*lpmgpu_detail::member_slot<lpmgpu_detail::ElasticCriticalStrain>::ptr;
        }
        else if (auto *ed = dynamic_cast<ParticleElasticDamage<nlayer> *>(pts[0]))
        {
            // setParticleProperty's k0, k1, damage threshold (particle_elastic_damage.h:28-29)
            d.ptype = LPMGPU_ELASTIC_DAMAGE;
            d.k0 = ed->k0;
            d.k1 = ed->k1;
            d.comp_tensile_ratio = ed->comp_tensile_ratio;
            d.damage_threshold = ed->damage_threshold;
        }
        else if (auto *hcf = dynamic_cast<ParticleFatigueHCF<nlayer> *>(pts[0]))
        {
            // the rate law and threshold of particle_fatigue_hcf.h:19-21
            d.ptype = LPMGPU_FATIGUE_HCF;
            d.E = hcf->E;
            d.mu = hcf->mu;
            d.fatigue_A = hcf->A;
            d.fatigue_B = hcf->B;
            d.fatigue_d = hcf->d;
            d.fatigue_limit_ratio = hcf->fatigue_limit_ratio;
            d.damage_threshold = hcf->damage_threshold;
        }
        else
            throw std::runtime_error("SolverStaticGPU: unsupported particle type");
        // the nonlocal neighbours Assembly::searchNonlocalNeighbors found (assembly.h:118-130), in
        // their list order, when the example ran the search
        std::vector<int32_t> nl_count(n, 0), nl_ids;
        for (auto *p : pts)
        {
            nl_count[p->id] = (int32_t)p->neighbors_nonlocal.size();
            for (auto *q : p->neighbors_nonlocal)
                nl_ids.push_back(q->id);
        }
        if (!nl_ids.empty())
        {
            d.nonlocal_count = nl_count.data();
            d.nonlocal_ids = nl_ids.data();
        }
        d.nonlocal_L = pts[0]->nonlocal_L;
        d.undamaged_type = undamaged_pt_type;
        d.max_iter = max_NR_iter;
        d.tol_iter = tol_NR_iter;
        d.cg_rtol = cg_rtol_;
        d.cg_atol = cg_atol_;
        d.precision = precision_;
        d.device = device_;
        d.direct = direct_;
        d.bond_nb0 = nb0.data();
        d.bond_nb1 = nb1.data();
        d.bond_p2 = p2.data();
        d.bond_kn = kn.data();
        d.bond_tv = tv.data();
        d.bond_damage = dmg.data();
        if (h_)
        {
            lpmgpu_destroy(h_);
            h_ = nullptr;
        }
        lpmgpu_detail::check(lpmgpu_create(&d, &h_), "lpmgpu_create");
    }

    void ensure_tolerances()
    {
        if (rebuild_needed_)
        {
            create(precision_, device_);
            rebuild_needed_ = false;
        }
    }

    void write_back()
    {
        auto &pts = ass.pt_sys;
        const size_t n = pts.size();
        lpmgpu_sizes sz{};
        lpmgpu_detail::check(lpmgpu_get_sizes(h_, &sz), "lpmgpu_get_sizes");
        const int nsv = (int)pts[0]->state_var.size();
        std::vector<double> xyz(3 * n), pin(3 * n), stress(6 * n), dmg(n), dmgv(n), sv((size_t)nsv * n),
            bd((size_t)sz.nbonds);
        lpmgpu_detail::check(lpmgpu_read_state(h_, xyz.data(), pin.data(), stress.data(), dmg.data(), dmgv.data(),
                                               sv.data(), bd.data()),
                             "lpmgpu_read_state");
        size_t b = 0;
        for (auto *p : pts)
        {
            const size_t i = (size_t)p->id;
            for (int k = 0; k < 3; ++k)
            {
                p->xyz[k] = xyz[3 * i + k];
                p->Pin[k] = pin[3 * i + k];
            }
            p->stress.assign(stress.begin() + 6 * i, stress.begin() + 6 * i + 6);
            p->damage = dmg[i];
            p->damage_visual = dmgv[i];
            for (int k = 0; k < nsv; ++k)
                p->state_var[k] = sv[(size_t)nsv * i + k];
        }
        for (auto *p : pts)
            for (int l = 0; l < nlayer; ++l)
                for (auto *bond : p->bond_layers[l])
                    bond->bdamage = bd[b++];
    }

    void export_K()
    {
        lpmgpu_sizes sz{};
        lpmgpu_detail::check(lpmgpu_get_sizes(h_, &sz), "lpmgpu_get_sizes");
        const size_t n = (size_t)sz.n, nnz = (size_t)sz.nnz_upper;
        std::vector<int64_t> kp(n + 1), ik((size_t)sz.dim * n + 1), jk(nnz);
        stiffness.kv.resize(nnz);
        lpmgpu_detail::check(lpmgpu_export_ref_csr(h_, kp.data(), ik.data(), jk.data(), stiffness.kv.data()),
                             "lpmgpu_export_ref_csr");
        stiffness.kp.assign(kp.begin(), kp.end());
        stiffness.ik.assign(ik.begin(), ik.end());
        stiffness.jk.assign(jk.begin(), jk.end());
        stiffness.K_pointer = stiffness.kp.data();
        stiffness.IK = stiffness.ik.data();
        stiffness.JK = stiffness.jk.data();
        stiffness.K_global = stiffness.kv.data();
    }
};
