// SolverFatigueGPU<nlayer>: a drop-in for LPM-CPP's SolverFatigue<nlayer> (include/solver_fatigue.h)
// on the device library, next to SolverStaticGPU (solver_static_gpu.h), whose problem packing and
// write-back it shares.  Include it after the LPM-CPP headers an example uses (it includes
// load_step_fatigue.h itself) and link liblpmgpu.so.
#pragma once

#include <cmath>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "load_step_fatigue.h"
#include "solver_static_gpu.h"

// SolverFatigueGPU<nlayer>: the same one-line switch for LPM-CPP's SolverFatigue<nlayer>
// (include/solver_fatigue.h:19-38), constructor arguments unchanged:
//
//     SolverFatigue<n_layer> solv_fatigue{undamaged_pt_type, pt_ass, StiffnessMode::Analytical,
//                                         SolverMode::CG, TimeMapMode::Linear, tau, dumpFile, max_iter, tol_iter};
//  -> SolverFatigueGPU<n_layer> solv_fatigue{...same arguments...};
//
// Every step of a cycle (BCs, stiffness, Newton), the particles' energy updates and the fatigue
// damage run on the device; the load spectrum, the cycle loop and the dN/dt time map stay on
// the host as in the reference.  Particle fields are written back after every static step and
// every cycle, before the dump.
template <int nlayer>
class SolverFatigueGPU : public SolverStaticGPU<nlayer>
{
public:
    TimeMapMode t_mode;
    double tau{0};
    std::vector<double> load_spectrum;

    SolverFatigueGPU(const int &p_undamaged, Assembly<nlayer> &p_ass, const StiffnessMode &p_stiff_mode,
                     const SolverMode &p_sol_mode, const TimeMapMode &p_t_mode, const double &p_tau,
                     const std::string &p_dumpFile, const int &p_niter, const double &p_tol,
                     int precision = LPMGPU_FP64, int device = 0)
        : SolverStaticGPU<nlayer>{p_undamaged, p_ass, p_stiff_mode, p_sol_mode, p_dumpFile, p_niter, p_tol,
                                  precision, device},
          t_mode(p_t_mode), tau(p_tau)
    {
    }

    // SolverFatigue::readLoad (solver_fatigue.h:40-57); a missing file throws instead of exit(1)
    void readLoad(const std::string &loadFile)
    {
        FILE *fpt = std::fopen(loadFile.c_str(), "r");
        if (!fpt)
            throw std::runtime_error("'" + loadFile + "' does not exist!");
        double data;
        while (std::fscanf(fpt, "%lf", &data) > 0)
            load_spectrum.push_back(data);
        std::fclose(fpt);
    }

    // SolverFatigue::generateLoadCycle (solver_fatigue.h:128-180)
    std::vector<LoadStep<nlayer>> generateLoadCycle(FatigueLoadType ltype, int N, int n_interval,
                                                    std::vector<std::vector<Particle<nlayer> *>> pt_groups)
    {
        const double f_0{load_spectrum[2 * N]}, f_1{load_spectrum[2 * N + 1]}, f_2{load_spectrum[2 * N + 2]};
        std::vector<LoadStep<nlayer>> load_cycle;
        for (int half = 0; half < 2; ++half)
        {
            const double v = half == 0 ? (f_1 - f_0) / n_interval : (f_2 - f_1) / n_interval;
            for (int i = 0; i < n_interval; ++i)
            {
                if (ltype == FatigueLoadType::LoadUniaxialDisp)
                    load_cycle.push_back(LoadUniaxialDisp<nlayer>(v, pt_groups[0], pt_groups[1], pt_groups[2]));
                if (ltype == FatigueLoadType::LoadUniaxialForce)
                    load_cycle.push_back(LoadUniaxialForce<nlayer>(v, pt_groups[0], pt_groups[1], pt_groups[2]));
                if (ltype == FatigueLoadType::LoadDogBoneDisp)
                    load_cycle.push_back(LoadDogBoneDisp<nlayer>(0, v, 0, pt_groups[0], pt_groups[1]));
                if (ltype == FatigueLoadType::LoadCTForce)
                    load_cycle.push_back(LoadCTForce<nlayer>(v, pt_groups[0], pt_groups[1], pt_groups[2]));
            }
        }
        return load_cycle;
    }

    // SolverFatigue::updateFatigueDamage (solver_fatigue.h:76-126)
    bool updateFatigueDamage(double dNdt)
    {
        int32_t any = 0;
        lpmgpu_detail::check(lpmgpu_fatigue_update_damage(this->h_, dNdt, &any), "lpmgpu_fatigue_update_damage");
        this->write_back();
        return any != 0;
    }

    // SolverFatigue::solveProblemStep (solver_fatigue.h:278-302)
    bool solveProblemStep(LoadStep<nlayer> &load_step)
    {
        this->ensure_tolerances();
        typename SolverStaticGPU<nlayer>::CStep c(load_step);
        lpmgpu_stats st{};
        const int32_t r = lpmgpu_fatigue_solve_step(this->h_, &c.step, &st);
        if (r != LPMGPU_OK && r != LPMGPU_ERR_NEWTON)
            lpmgpu_detail::check(r, "lpmgpu_fatigue_solve_step");
        tally(st);
        return r == LPMGPU_OK;
    }

    // SolverFatigue::solveProblemOneCycle (solver_fatigue.h:221-241), one device call
    void solveProblemOneCycle(std::vector<LoadStep<nlayer>> &load, double dNdt)
    {
        this->ensure_tolerances();
        std::vector<typename SolverStaticGPU<nlayer>::CStep> cs;
        cs.reserve(load.size());
        for (auto &l : load)
            cs.emplace_back(l);
        std::vector<lpmgpu_load_step> steps;
        for (auto &c : cs)
            steps.push_back(c.step);
        lpmgpu_stats st{};
        int32_t any = 0;
        lpmgpu_detail::check(lpmgpu_fatigue_cycle(this->h_, steps.data(), (int32_t)steps.size(), dNdt, &st, &any),
                             "lpmgpu_fatigue_cycle");
        tally(st);
        this->write_back();
    }

    // SolverFatigue::solveProblemCyclic (solver_fatigue.h:183-218)
    void solveProblemCyclic(FatigueLoadType loadType, int n_interval,
                            std::vector<std::vector<Particle<nlayer> *>> pt_groups)
    {
        const double n_cycles = 0.5 * (load_spectrum.size() - 1);
        double t{0}, dNdt{1};
        int N{0};
        do
        {
            printf("Cycle-%d starts:\n\n", N + 1);
            std::vector<LoadStep<nlayer>> load_cycle = generateLoadCycle(loadType, N, n_interval, pt_groups);
            dNdt = (t_mode == TimeMapMode::Linear) ? (int)(1 / tau) : (int)(1 / tau * exp(t++ / tau));
            solveProblemOneCycle(load_cycle, dNdt);
            N += (int)dNdt;
            if (!this->dumpFile.empty())
                this->ass.writeDump(this->dumpFile, N);
        } while (N < n_cycles);
        if (this->export_stiffness)
            this->export_K();
    }

    // SolverFatigue::solveProblemStatic (solver_fatigue.h:244-275)
    void solveProblemStatic(std::vector<LoadStep<nlayer>> &load, int &start_index)
    {
        int n_step = (int)load.size();
        for (int i = 0; i < n_step; i++)
        {
        restart:
            printf("Loading step-%d, iteration starts:\n", i + start_index);
            const bool is_converged = solveProblemStep(load[i]);
            if (!is_converged)
            {
                lpmgpu_detail::check(lpmgpu_reset_state(this->h_), "lpmgpu_reset_state");
                load[i].loadCutHalf();
                load.insert(load.begin() + i, load[i]);
                ++n_step;
                printf("Step-%d not converging\n\n", i + start_index);
                goto restart;
            }
            lpmgpu_detail::check(lpmgpu_update_state_var(this->h_), "lpmgpu_update_state_var");
            lpmgpu_detail::check(lpmgpu_store_state(this->h_), "lpmgpu_store_state");
            this->write_back();
            if (!this->dumpFile.empty())
                this->ass.writeDump(this->dumpFile, i);
        }
        start_index += n_step;
        if (this->export_stiffness)
            this->export_K();
    }

private:
    void tally(const lpmgpu_stats &st)
    {
        this->totals.newton_solves += st.newton_solves;
        this->totals.cg_iters += st.cg_iters;
        this->totals.cg_maxit_hits += st.cg_maxit_hits;
        this->totals.direct_solves += st.direct_solves;
        this->reaction_force.assign(1, st.reaction_norm);
    }
};
