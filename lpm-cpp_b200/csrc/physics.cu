// Per-Newton-iteration particle physics on the device, one thread per particle, each bond
// loop in the reference's list order so the sums round exactly as the reference does:
//   Particle::updateBondsGeometry / Bond::updatebGeometry  include/particle.h:164-181, bond.h:30-39
//   ParticleElastic::updateBondsForce                      include/particle_elastic.h:38-50
//   ParticleJ2Plasticity::updateBondsForce                 include/particle_j2plasticity.h:63-76
//   ParticleElasticDamage::updateBondsForce                include/particle_elastic_damage.h:80-91
//   Particle::updateParticleForce / Stress / DamageVisual  include/particle.h:151-240
//   Solver::updateRR                                       include/solver.h:112-126
//   ParticleJ2Plasticity::updateParticleStateVariables     include/particle_j2plasticity.h:78-140
//   SolverStatic::updateStaticDamage                       include/solver_static.h:32-62
//   Solver::updateForceBC / updateDisplacementBC           include/solver.h:129-188
// The reference finds the opposite bond with a linear find_if per bond (particle.h:207);
// here it is the precomputed brev index.
#include "lpm_internal.cuh"

namespace lpm
{

struct PhysArgs
{
    int n, dim, ptype;
    const int *__restrict__ bstart, *__restrict__ nb0, *__restrict__ bp2, *__restrict__ brev;
    double *__restrict__ xyz;
    const double *__restrict__ dis0, *__restrict__ Kn, *__restrict__ Tv;
    double *__restrict__ dis, *__restrict__ dLe, *__restrict__ dLp, *__restrict__ bstrain, *__restrict__ cs;
    double *__restrict__ bforce, *__restrict__ bdamage;
    double *__restrict__ dLe_total, *__restrict__ TdLe_total, *__restrict__ cs_sum;
    const double *__restrict__ damage;
};

// Sequential sum of v over lanes 0 .. cnt-1 in lane order, the same in every lane: the bond
// loop's own accumulation order, so the result rounds exactly as the reference's loop does.
__device__ __forceinline__ double lane_ordered_sum(double acc, double v, int cnt)
{
    for (int k = 0; k < cnt; ++k)
        acc += __shfl_sync(0xffffffffu, v, k);
    return acc;
}

// updateBondsGeometry + updateBondsForce: one warp per particle, lane k on the k-th bond of a
// 32-bond chunk of one layer's list.  Every per-bond array is read and written contiguously by
// the warp (coalesced); only the partner's coordinates and damage are gathers.  The layer sums
// (dLe, Tv*dLe, cosines) are taken in bond order through the lanes, as the reference's loop
// takes them (particle.h:164-181).
constexpr int kPhysWarps = 8;
__global__ void __launch_bounds__(32 * kPhysWarps) k_geometry_force(PhysArgs a)
{
    const int lane = threadIdx.x & 31;
    const int nw = gridDim.x * kPhysWarps;
    const bool dmg_max = a.ptype == LPMGPU_J2 || a.ptype == LPMGPU_ELASTIC_DAMAGE || a.ptype == LPMGPU_FATIGUE_HCF;
    for (int i = blockIdx.x * kPhysWarps + (threadIdx.x >> 5); i < a.n; i += nw)
    {
        const int b0 = a.bstart[i], b1 = b0 + a.nb0[i], be = a.bstart[i + 1];
        const double xi0 = a.xyz[3 * i], xi1 = a.xyz[3 * i + 1], xi2 = a.xyz[3 * i + 2];
        double dlt[2];
        for (int L = 0; L < 2; ++L)
        {
            const int lo = L == 0 ? b0 : b1, hi = L == 0 ? b1 : be;
            double s = 0, ts = 0, cx = 0, cy = 0, cz = 0;
            for (int c0 = lo; c0 < hi; c0 += 32)
            {
                const int b = c0 + lane, cnt = min(32, hi - c0);
                double dle = 0, tdle = 0, c[3] = {0, 0, 0};
                if (b < hi)
                {
                    const int j = a.bp2[b];
                    const double dx = xi0 - a.xyz[3 * j], dy = xi1 - a.xyz[3 * j + 1], dz = xi2 - a.xyz[3 * j + 2];
                    const bool broken = fabs(a.bdamage[b] - 1.0) < kEps;
                    const double dis = sqrt(dx * dx + dy * dy + dz * dz);
                    const double d0 = a.dis0[b];
                    const double dL = broken ? 0.0 : (dis - d0);
                    const double bst = broken ? 0.0 : (dL / dis);
                    dle = broken ? 0.0 : (dis - d0 - a.dLp[b]);
                    c[0] = broken ? 0.0 : (dx / dis);
                    c[1] = broken ? 0.0 : (dy / dis);
                    c[2] = broken ? 0.0 : (dz / dis);
                    a.dis[b] = dis;
                    a.bstrain[b] = bst;
                    a.dLe[b] = dle;
                    a.cs[3 * (int64_t)b] = c[0];
                    a.cs[3 * (int64_t)b + 1] = c[1];
                    a.cs[3 * (int64_t)b + 2] = c[2];
                    tdle = a.Tv[b] * dle;
                }
                s = lane_ordered_sum(s, dle, cnt);
                ts = lane_ordered_sum(ts, tdle, cnt);
                cx = lane_ordered_sum(cx, c[0], cnt);
                cy = lane_ordered_sum(cy, c[1], cnt);
                cz = lane_ordered_sum(cz, c[2], cnt);
            }
            dlt[L] = s;
            if (lane == 0)
            {
                a.dLe_total[2 * i + L] = s;
                a.TdLe_total[2 * i + L] = ts;
                a.cs_sum[6 * i + 3 * L] = cx;
                a.cs_sum[6 * i + 3 * L + 1] = cy;
                a.cs_sum[6 * i + 3 * L + 2] = cz;
            }
        }
        __syncwarp(); // dLe of a bond is read below by another lane than the one that wrote it
        const double di = a.damage[i];
        for (int b = b0 + lane; b < be; b += 32)
        {
            const int L = b < b1 ? 0 : 1;
            double f = 2. * a.Kn[b] * a.dLe[b] + 2. * a.Tv[b] * dlt[L];
            double D = a.bdamage[b];
            if (dmg_max)
            {
                D = std_max(D, std_max(di, a.damage[a.bp2[b]]));
                a.bdamage[b] = D;
            }
            f *= (1.0 - D);
            a.bforce[b] = f;
        }
    }
}

struct ForceArgs
{
    int n, dim, nneighbors;
    double pvol;
    const int *__restrict__ bstart, *__restrict__ brev, *__restrict__ nb, *__restrict__ cons;
    const double *__restrict__ cs, *__restrict__ dis, *__restrict__ bforce, *__restrict__ bdamage,
        *__restrict__ pex;
    double *__restrict__ pin, *__restrict__ stress, *__restrict__ damage_visual, *__restrict__ res;
    double *__restrict__ partials; // [grid][2]: residual^2, reaction^2
};

__device__ __forceinline__ double warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// deterministic block sum (fixed tree), result valid in thread 0
template <int NT>
__device__ __forceinline__ double block_sum(double v, double *sh)
{
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0)
        sh[w] = v;
    __syncthreads();
    double r = 0;
    if (w == 0)
    {
        r = (l < NT / 32) ? sh[l] : 0.0;
        r = warp_sum(r);
    }
    __syncthreads();
    return r;
}

// updateParticleForce + updateParticleStress + updateParticleDamageVisual, then updateRR: one warp
// per particle, lanes over the bond list in 32-bond chunks (coalesced per-bond reads; the
// opposite bond's force is a gather), sums in bond order through the lanes.  The per-block
// partials of the residual and reaction norms are summed in a fixed order (each warp over its
// particles in turn, then the warps in order), so every run rounds alike.
constexpr int kForceWarps = 8;
__global__ void __launch_bounds__(32 * kForceWarps) k_internal_force(ForceArgs a)
{
    __shared__ double sh[2 * kForceWarps];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nw = gridDim.x * kForceWarps;
    double rsq = 0.0, rea = 0.0; // this warp's sums (valid in lane 0)
    for (int i = blockIdx.x * kForceWarps + w; i < a.n; i += nw)
    {
        const int b0 = a.bstart[i], be = a.bstart[i + 1];
        const int nbi = a.nb[i];
        const double V_m = a.pvol * nbi / a.nneighbors;
        double P0 = 0., P1 = 0., P2 = 0.;
        double S0 = 0, S1 = 0, S2 = 0, S3 = 0, S4 = 0, S5 = 0, dv = 0;
        for (int c0 = b0; c0 < be; c0 += 32)
        {
            const int b = c0 + lane, cnt = min(32, be - c0);
            double p0 = 0, p1 = 0, p2 = 0, s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0, s5 = 0, dmg = 0;
            if (b < be)
            {
                const double fs = a.bforce[b] + a.bforce[a.brev[b]];
                const double cx = a.cs[3 * (int64_t)b], cy = a.cs[3 * (int64_t)b + 1], cz = a.cs[3 * (int64_t)b + 2];
                p0 = cx * 0.5 * fs;
                p1 = cy * 0.5 * fs;
                p2 = cz * 0.5 * fs;
                const double wgt = 0.5 / V_m * (a.dis[b]) * 0.5 * fs;
                s0 = wgt * (cx) * (cx);
                s1 = wgt * (cy) * (cy);
                s2 = wgt * (cz) * (cz);
                s3 = wgt * (cy) * (cz);
                s4 = wgt * (cx) * (cz);
                s5 = wgt * (cx) * (cy);
                dmg = a.bdamage[b];
            }
            P0 = lane_ordered_sum(P0, p0, cnt);
            P1 = lane_ordered_sum(P1, p1, cnt);
            P2 = lane_ordered_sum(P2, p2, cnt);
            S0 = lane_ordered_sum(S0, s0, cnt);
            S1 = lane_ordered_sum(S1, s1, cnt);
            S2 = lane_ordered_sum(S2, s2, cnt);
            S3 = lane_ordered_sum(S3, s3, cnt);
            S4 = lane_ordered_sum(S4, s4, cnt);
            S5 = lane_ordered_sum(S5, s5, cnt);
            dv = lane_ordered_sum(dv, dmg, cnt);
        }
        if (lane == 0)
        {
            a.pin[3 * i] = P0;
            a.pin[3 * i + 1] = P1;
            a.pin[3 * i + 2] = P2;
            double *st = a.stress + 6 * (int64_t)i;
            st[0] = S0;
            st[1] = S1;
            st[2] = S2;
            st[3] = S3;
            st[4] = S4;
            st[5] = S5;
            a.damage_visual[i] = dv / (double)nbi;
            const double P[3] = {P0, P1, P2};
            for (int k = 0; k < a.dim; ++k)
            {
                const int c = a.cons[3 * i + k];
                const double v = (1 - c) * (a.pex[3 * i + k] - P[k]);
                a.res[(int64_t)a.dim * i + k] = v;
                rsq += v * v;
                if (c == 1)
                    rea += P[k] * P[k];
            }
        }
    }
    if (lane == 0)
    {
        sh[w] = rsq;
        sh[kForceWarps + w] = rea;
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double r = 0, q = 0;
        for (int k = 0; k < kForceWarps; ++k)
        {
            r += sh[k];
            q += sh[kForceWarps + k];
        }
        a.partials[2 * blockIdx.x] = r;
        a.partials[2 * blockIdx.x + 1] = q;
    }
}

// fixed-order sum of the per-block partials; accumulates the reaction history
__global__ void k_finalize_rr(int nblk, const double *__restrict__ partials, Scalars *scal, int accumulate)
{
    __shared__ double sh[32];
    double r = 0, q = 0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x)
    {
        r += partials[2 * b];
        q += partials[2 * b + 1];
    }
    const double R = block_sum<256>(r, sh);
    const double Q = block_sum<256>(q, sh);
    if (threadIdx.x == 0)
    {
        scal->res_sq = R;
        if (accumulate)
            scal->reaction_sq += Q;
    }
}

// grid of the warp-per-particle kernels: one warp per particle up to 16 blocks of 8 warps per SM;
// beyond that each warp takes several particles
static int phys_grid(const Problem &p)
{
    // the partials buffer holds 2 x kMaxGridBlocks doubles
    const int64_t cap = std::min<int64_t>((int64_t)p.num_sms * 16, kMaxGridBlocks);
    return (int)std::max<int64_t>(1, std::min<int64_t>(div_up(p.n, kPhysWarps), cap));
}

cudaError_t launch_geometry_force(Problem &p)
{
    PhysArgs a;
    a.n = p.n;
    a.dim = p.dim;
    a.ptype = p.desc.ptype;
    a.bstart = p.bstart;
    a.nb0 = p.nb0;
    a.bp2 = p.bp2;
    a.brev = p.brev;
    a.xyz = p.xyz;
    a.dis0 = p.dis0;
    a.Kn = p.Kn;
    a.Tv = p.Tv;
    a.dis = p.dis;
    a.dLe = p.dLe;
    a.dLp = p.dLp;
    a.bstrain = p.bstrain;
    a.cs = p.cs;
    a.bforce = p.bforce;
    a.bdamage = p.bdamage;
    a.dLe_total = p.dLe_total;
    a.TdLe_total = p.TdLe_total;
    a.cs_sum = p.cs_sum;
    a.damage = p.damage;
    k_geometry_force<<<phys_grid(p), 32 * kPhysWarps, 0, p.stream>>>(a);
    p.ctr.kernel_launches++;
    return cudaGetLastError();
}

// accumulate_reaction: Solver::updateRR appends the reaction forces to the history
// (solver.h:122-123); Assembly::updateForceState alone (solver_static.h:132-133) does not
cudaError_t launch_update_rr_impl(Problem &p, bool accumulate_reaction)
{
    ForceArgs a;
    a.n = p.n;
    a.dim = p.dim;
    a.nneighbors = p.cell.nneighbors;
    a.pvol = p.cell.pvol;
    a.bstart = p.bstart;
    a.brev = p.brev;
    a.nb = p.nb;
    a.cons = p.cons;
    a.cs = p.cs;
    a.dis = p.dis;
    a.bforce = p.bforce;
    a.bdamage = p.bdamage;
    a.pex = p.pex;
    a.pin = p.pin;
    a.stress = p.stress;
    a.damage_visual = p.damage_visual;
    a.res = p.res;
    a.partials = p.partials;
    const int nblk = phys_grid(p);
    k_internal_force<<<nblk, 32 * kForceWarps, 0, p.stream>>>(a);
    k_finalize_rr<<<1, 256, 0, p.stream>>>(nblk, p.partials, p.scal, accumulate_reaction ? 1 : 0);
    p.ctr.kernel_launches += 2;
    return cudaGetLastError();
}

// ParticleJ2Plasticity::updateParticleStateVariables (particle_j2plasticity.h:78-140)
__global__ void k_j2_update(int n, double E, double mu, double sigmay, double xi, double H, double A,
                            const int *__restrict__ bstart, const double *__restrict__ stress,
                            const double *__restrict__ dis, const double *__restrict__ cs, double *__restrict__ sv,
                            double *__restrict__ dLp, double *__restrict__ ddot_local)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    double *s = sv + 7 * (int64_t)i;
    double st[6], dpl[6] = {0, 0, 0, 0, 0, 0};
    double sigma_eq = 0.0, triax = 0.0, dlambda = 0.0;
    for (int j = 0; j < 6; ++j)
        st[j] = stress[6 * (int64_t)i + j];
    const double sigma_m = 1.0 / 3.0 * (st[0] + st[1] + st[2]);
    for (int j = 0; j < 3; j++)
        st[j] -= sigma_m;
    for (int j = 0; j < 6; j++)
        st[j] -= s[j + 1];
    for (int j = 0; j < 6; j++)
    {
        if (j < 3)
            sigma_eq += st[j] * st[j];
        else
            sigma_eq += 2.0 * st[j] * st[j];
    }
    sigma_eq = sqrt(3.0 / 2.0 * sigma_eq);
    const double yield = sigma_eq - (sigmay + (1.0 - xi) * H * s[0]);
    const double G = E / 2 / (1 + mu);
    if (yield > 0.0)
        dlambda = yield / (3 * G + H);
    s[0] += dlambda;
    for (int j = 0; j < 6; j++)
        if (fabs(sigma_eq) > kEps)
        {
            dpl[j] = dlambda * 1.5 * st[j] / sigma_eq;
            s[j + 1] += 2. / 3. * xi * H * dpl[j];
        }
    for (int b = bstart[i]; b < bstart[i + 1]; ++b)
    {
        const double cx = cs[3 * (int64_t)b], cy = cs[3 * (int64_t)b + 1], cz = cs[3 * (int64_t)b + 2];
        const double ddLp = dis[b] * (dpl[0] * cx * cx + dpl[1] * cy * cy + dpl[2] * cz * cz + 2 * dpl[3] * cy * cz +
                                      2 * dpl[4] * cx * cz + 2 * dpl[5] * cx * cy);
        dLp[b] += ddLp;
    }
    if (sigma_eq > kEps)
        triax = sigma_m / sigma_eq;
    ddot_local[i] = dlambda * (1.0 + A * triax);
}

cudaError_t launch_update_state_var(Problem &p)
{
    if (p.desc.ptype == LPMGPU_ELASTIC_DAMAGE)
        return launch_edamage_update(p);
    if (p.desc.ptype == LPMGPU_FATIGUE_HCF)
        return launch_hcf_update(p);
    if (p.desc.ptype != LPMGPU_J2)
        return cudaSuccess;
    k_j2_update<<<div_up(p.n, 128), 128, 0, p.stream>>>(p.n, p.desc.E, p.desc.mu, p.desc.sigmay, p.desc.xi, p.desc.H,
                                                        p.desc.A, p.bstart, p.stress, p.dis, p.cs, p.sv, p.dLp,
                                                        p.ddot_local);
    p.ctr.kernel_launches++;
    return cudaGetLastError();
}

// SolverStatic::updateStaticDamage.  The nonlocal rate comes from k_nonlocal_average when a
// nonlocal search ran; without one it is 0/0 (solver_static.h:39-51), exactly as in the reference
// when searchNonlocalNeighbors was not called.  Elastic particles ignore it; J2 and elastic-damage
// particles add it to their damage and set the damage to 1 at their threshold
// (particle_j2plasticity.h:142-152, particle_elastic_damage.h:172-181).
__global__ void k_static_damage(int n, int ptype, int undamaged, double critical, double threshold,
                                const int *__restrict__ type, const int *__restrict__ bstart,
                                const double *__restrict__ bstrain, const double *__restrict__ ddot_nl,
                                double *__restrict__ bdamage, double *__restrict__ damage,
                                const double *__restrict__ damage_last, Scalars *scal)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || type[i] == undamaged)
        return;
    bool changed = false;
    if (ptype == LPMGPU_J2 || ptype == LPMGPU_ELASTIC_DAMAGE)
    {
        volatile double zero = 0.0;
        const double ddot_nonlocal = ddot_nl ? ddot_nl[i] : zero / zero;
        double d = damage[i] + ddot_nonlocal;
        if (d >= threshold)
            d = 1;
        damage[i] = d;
        changed = fabs(d - damage_last[i]) > 1e-3;
    }
    else
    {
        for (int b = bstart[i]; b < bstart[i + 1]; ++b)
            if (bstrain[b] >= critical && fabs(bdamage[b] - 1.0) > kEps)
            {
                changed = true;
                bdamage[b] = 1;
            }
    }
    if (changed)
        atomicExch(&scal->any_flag, 1);
}

cudaError_t launch_static_damage(Problem &p)
{
    cudaError_t e = cudaMemsetAsync(&p.scal->any_flag, 0, sizeof(int), p.stream);
    if (e != cudaSuccess)
        return e;
    // fatigue particles keep Particle::updateParticleStaticDamage, which changes nothing
    // (particle.h:63): their damage moves only in SolverFatigue::updateFatigueDamage
    if (p.desc.ptype == LPMGPU_FATIGUE_HCF)
        return cudaSuccess;
    if (p.desc.ptype != LPMGPU_ELASTIC && (e = launch_nonlocal_average(p)) != cudaSuccess)
        return e;
    // damage_threshold is never assigned for J2 (particle_j2plasticity.h:22): 0
    const double threshold = (p.desc.ptype == LPMGPU_ELASTIC_DAMAGE) ? p.desc.damage_threshold : 0.0;
    k_static_damage<<<div_up(p.n, 128), 128, 0, p.stream>>>(p.n, p.desc.ptype, p.desc.undamaged_type,
                                                            p.desc.critical_bstrain, threshold, p.type, p.bstart,
                                                            p.bstrain, p.ddot_nonlocal, p.bdamage, p.damage,
                                                            p.damage_last, p.scal);
    p.ctr.kernel_launches++;
    return cudaGetLastError();
}

// Solver::solveLinearSystem position update (solver.h:101-108)
__global__ void k_add_disp(int n, int dim, const double *__restrict__ x, double *__restrict__ xyz)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    for (int k = 0; k < dim; ++k)
        xyz[3 * i + k] = xyz[3 * i + k] + (0.0 + x[(int64_t)dim * i + k]);
}

cudaError_t launch_add_disp(Problem &p)
{
    k_add_disp<<<div_up(p.n, 256), 256, 0, p.stream>>>(p.n, p.dim, p.x, p.xyz);
    p.ctr.kernel_launches++;
    return cudaGetLastError();
}

__global__ void k_force_bc(int count, const int *__restrict__ ids, double fx, double fy, double fz,
                           double *__restrict__ pex)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= count)
        return;
    const int i = ids[q];
    pex[3 * i] += fx / count;
    pex[3 * i + 1] += fy / count;
    pex[3 * i + 2] += fz / count;
}

__global__ void k_disp_bc(int count, const int *__restrict__ ids, int flag, double step, double *__restrict__ xyz,
                          int *__restrict__ cons)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= count)
        return;
    const int i = ids[q];
    xyz[3 * i + flag] = xyz[3 * i + flag] + step;
    cons[3 * i + flag] = 1;
}

// updateForceBC then updateDisplacementBC, each BC in order.  A particle that appears twice in
// one group would be updated by two threads; the reference's groups hold distinct particles.
cudaError_t launch_apply_bc(Problem &p, const lpmgpu_load_step &s)
{
    size_t total = 0;
    for (int f = 0; f < s.nforce; ++f)
        total += (size_t)s.force[f].count;
    for (int d = 0; d < s.ndisp; ++d)
        total += (size_t)s.disp[d].count;
    if (total == 0)
        return cudaSuccess;
    int *dids = nullptr;
    cudaError_t e = cudaMallocAsync(&dids, sizeof(int) * total, p.stream);
    if (e != cudaSuccess)
        return e;
    std::vector<int> h(total);
    size_t o = 0;
    for (int f = 0; f < s.nforce; ++f)
        for (int q = 0; q < s.force[f].count; ++q)
            h[o++] = s.force[f].ids[q];
    for (int d = 0; d < s.ndisp; ++d)
        for (int q = 0; q < s.disp[d].count; ++q)
            h[o++] = s.disp[d].ids[q];
    e = cudaMemcpyAsync(dids, h.data(), sizeof(int) * total, cudaMemcpyHostToDevice, p.stream);
    o = 0;
    for (int f = 0; f < s.nforce && e == cudaSuccess; ++f)
    {
        const auto &b = s.force[f];
        if (b.count > 0)
        {
            k_force_bc<<<div_up(b.count, 256), 256, 0, p.stream>>>(b.count, dids + o, b.fx, b.fy, b.fz, p.pex);
            p.ctr.kernel_launches++;
        }
        o += b.count;
    }
    for (int d = 0; d < s.ndisp && e == cudaSuccess; ++d)
    {
        const auto &b = s.disp[d];
        if (b.count > 0)
        {
            k_disp_bc<<<div_up(b.count, 256), 256, 0, p.stream>>>(b.count, dids + o, b.flag, b.step, p.xyz, p.cons);
            p.ctr.kernel_launches++;
        }
        o += b.count;
    }
    if (e == cudaSuccess)
        e = cudaGetLastError();
    // the host vector must outlive the async copy
    cudaError_t s2 = cudaStreamSynchronize(p.stream);
    cudaFreeAsync(dids, p.stream);
    return e != cudaSuccess ? e : s2;
}

} // namespace lpm
