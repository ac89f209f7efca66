// Serving loop: LPM solves (a problem description and its load path) are submitted while others
// run; each is admitted when its device memory fits an HBM budget, joins the running batch
// between two rounds (continuous batching: its CG iterations share the batched launches with
// every other running solve), and leaves it when its last load step is done.  Its state, K and
// Krylov vectors stay resident on the device from admission to completion.
//
// Two host threads per server:
//   admission  takes queued requests in arrival order while their estimated device memory fits
//              the budget, builds their device problems (lpmgpu_create) and hands them over;
//   worker     owns the batch: adds the handed-over problems, runs rounds, and for each member
//              that finished copies its final positions to the host, destroys its device problem
//              and returns its memory to the budget.
// Clients submit, poll, wait and fetch results from any thread.
#include <algorithm>
#include <cstdlib>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "lpm_internal.cuh"

namespace
{

using Clock = std::chrono::steady_clock;

struct OwnedStep
{
    std::vector<std::vector<int32_t>> dids, fids;
    std::vector<lpmgpu_dispbc> d;
    std::vector<lpmgpu_forcebc> f;
    lpmgpu_load_step view{};

    explicit OwnedStep(const lpmgpu_load_step &s)
    {
        for (int k = 0; k < s.ndisp; ++k)
        {
            dids.emplace_back(s.disp[k].ids, s.disp[k].ids + s.disp[k].count);
            d.push_back(s.disp[k]);
        }
        for (int k = 0; k < s.nforce; ++k)
        {
            fids.emplace_back(s.force[k].ids, s.force[k].ids + s.force[k].count);
            f.push_back(s.force[k]);
        }
        for (size_t k = 0; k < d.size(); ++k)
            d[k].ids = dids[k].data();
        for (size_t k = 0; k < f.size(); ++k)
            f[k].ids = fids[k].data();
        view = {d.data(), (int32_t)d.size(), f.data(), (int32_t)f.size()};
    }
};

struct Request
{
    int64_t id = 0;
    int32_t state = 0; // 0 queued, 1 running, 2 done, 3 failed
    int32_t status = LPMGPU_OK;
    lpmgpu_desc desc{};
    std::vector<double> xyz, kn, tv, bdmg;
    std::vector<int32_t> type, nb0, nb1, p2, nl_count, nl_ids;
    std::vector<OwnedStep> steps;
    // a fatigue request (lpmgpu_server_submit_fatigue): steps = nstatic static steps, then
    // ncycles cycles of cycle_len steps, cycle c with dN/dt dndt[c]
    bool fatigue = false;
    int32_t nstatic = 0, cycle_len = 0, ncycles = 0;
    std::vector<double> dndt;
    int64_t est_bytes = 0, bytes = 0;
    int64_t volume = 0; // bytes its CG streams per iteration (matrix values and block columns)
    int64_t counted = 0; // its share of the running volume (0 for a solo request)
    lpmgpu_solver *h = nullptr;
    int32_t member = -1;
    lpmgpu_member_info info{};
    std::vector<double> result; // n*3 final positions
    Clock::time_point t_submit, t_start, t_done;
};

// Device memory a problem is expected to take, before it exists (the admission test).  Per
// particle: the full symmetric block row (connections x d^2 values, FP64 and in mixed precision
// FP32, plus a column index per block), with slack for the sliced-ELL padding; per bond ~20
// doubles; vectors and particle state.  Connection and bond counts are upper values per lattice.
int64_t estimate_bytes(const lpmgpu_desc &d)
{
    int nc = 31, nb = 12, dim = 2;
    switch (d.lattice)
    {
    case LPMGPU_SQUARE2D: nc = 25; nb = 8; dim = 2; break;
    case LPMGPU_HEXAGON2D: nc = 31; nb = 12; dim = 2; break;
    case LPMGPU_SC3D: nc = 61; nb = 18; dim = 3; break;
    case LPMGPU_FCC3D: nc = 100; nb = 18; dim = 3; break;
    default: nc = 80; nb = 14; dim = 3; break;
    }
    const int64_t per_block = (int64_t)dim * dim * (8 + (d.precision == LPMGPU_MIXED ? 4 : 0)) + 4;
    // mixed: the FP32 Krylov vectors, three of them doubled for the batch's single-reduction CG
    const int64_t mixed_vec = d.precision == LPMGPU_MIXED ? (int64_t)dim * 9 * 4 : 0;
    int64_t per_particle = (int64_t)(1.25 * nc * per_block) + (int64_t)nb * 20 * 8 + 40 * 8 * dim + 512 + mixed_vec;
    // the fast assembly's lists: at most nb^2 two-hop paths of 5 bytes, a count per slot, T and
    // Ts per bond, U and the row offset per particle
    per_particle += (int64_t)nb * nb * 5 + nc + (int64_t)nb * 16 + 56;
    if (d.nonlocal_cutoff_ratio > 0 && d.radius > 0)
    {
        // nonlocal lists: the particles within cutoff_ratio x nonlocal_L, counted for the densest
        // packing of the dimension (hexagonal: 2 sqrt(3) r^2 per particle; FCC: 4 sqrt(2) r^3),
        // 4 bytes each, plus the list offset and the nonlocal rate of the particle
        const double R = d.nonlocal_cutoff_ratio * d.nonlocal_L, r = d.radius, pi = 3.14159265358979;
        const double m = (dim == 2) ? pi * R * R / (2 * std::sqrt(3.0) * r * r)
                                    : 4.0 / 3.0 * pi * R * R * R / (4 * std::sqrt(2.0) * r * r * r);
        per_particle += 4 * (int64_t)(1.2 * m + 8) + 12;
    }
    int64_t lists = 0;
    if (d.nonlocal_count && d.nonlocal_ids)
    {
        // the caller's nonlocal lists, counted exactly: 4 bytes an entry, an offset and a rate
        for (int i = 0; i < d.n; ++i)
            lists += 4 * (int64_t)std::max(0, d.nonlocal_count[i]);
        per_particle += 12;
    }
    return (int64_t)d.n * per_particle + lists + (8 << 20);
}

} // namespace

struct lpmgpu_server
{
    int device = 0;
    int64_t budget = 0;
    std::mutex mu;
    std::condition_variable cv_admit, cv_work, cv_done;
    std::deque<Request *> queue;
    std::vector<Request *> ready;
    std::map<int64_t, std::unique_ptr<Request>> reqs;
    std::vector<double> latencies;
    int64_t next_id = 1, used = 0, reserved = 0, peak = 0, running = 0, done = 0, failed = 0, submitted = 0;
    int64_t rounds = 0, finished_epoch = 0;
    int64_t slice = -1; // requested CG slice, applied by the worker between rounds (-1: unchanged)
    int32_t lanes = 0;  // requested batch lanes, applied by the worker once no request runs (0: unchanged)
    // Cap on the running requests' summed per-iteration matrix stream.  Past a few hundred MB the
    // batched CG already streams at HBM speed; more members running at once only share that
    // bandwidth, thrash L2 with their Krylov vectors and lengthen every round, so admitted
    // requests beyond the cap wait (a request that alone exceeds it runs when nothing else does;
    // smaller ones behind it may go first).  LPMGPU_SERVE_VOLUME_MB sets it.
    int64_t volume_cap = int64_t(768) << 20, running_volume = 0;
    // Solo requests (lpmgpu_batch_set_solo_bytes) solve alone between the batched launches, so
    // they do not count against the cap.  solo_request: a new value for the worker to apply.
    int64_t solo_bytes = 192000000, solo_request = -1;
    int64_t counted_volume(const Request *r) const
    {
        return (solo_bytes > 0 && r->volume >= solo_bytes) ? 0 : r->volume;
    }
    bool stop = false;
    int32_t worker_status = LPMGPU_OK;
    lpmgpu_batch *batch = nullptr;
    std::thread admit_thread, work_thread;
    Clock::time_point t0;

    double since(Clock::time_point t) const { return std::chrono::duration<double>(t - t0).count(); }

    void admission()
    {
        cudaSetDevice(device);
        for (;;)
        {
            Request *r = nullptr;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_admit.wait(lk, [&] {
                    if (stop)
                        return true;
                    if (queue.empty())
                        return false;
                    const int64_t need = queue.front()->est_bytes;
                    // a request larger than the whole budget runs alone
                    return used + reserved + need <= budget || (used + reserved == 0 && running == 0);
                });
                if (stop)
                    return;
                r = queue.front();
                queue.pop_front();
                reserved += r->est_bytes;
            }
            lpmgpu_solver *h = nullptr;
            const int32_t s = lpmgpu_create(&r->desc, &h);
            lpmgpu_sizes sz{};
            if (s == LPMGPU_OK)
                lpmgpu_get_sizes(h, &sz);
            std::unique_lock<std::mutex> lk(mu);
            reserved -= r->est_bytes;
            if (s == LPMGPU_ERR_OUT_OF_MEMORY && (running > 0 || !ready.empty()))
            {
                // the estimate was low: wait for a running solve to finish, then try again
                queue.push_front(r);
                const int64_t ep = finished_epoch;
                cv_admit.wait(lk, [&] { return stop || finished_epoch != ep; });
                continue;
            }
            if (s != LPMGPU_OK)
            {
                r->state = 3;
                r->status = s;
                r->t_done = Clock::now();
                failed++;
                cv_done.notify_all();
                continue;
            }
            r->h = h;
            r->bytes = sz.device_bytes;
            r->volume = lpm::cg_stream_bytes(h->p);
            used += r->bytes;
            peak = std::max(peak, used);
            // the description's host arrays were only needed by lpmgpu_create
            r->xyz.clear();
            r->xyz.shrink_to_fit();
            r->type.clear();
            r->nb0.clear();
            r->nb1.clear();
            r->p2.clear();
            r->kn.clear();
            r->tv.clear();
            r->bdmg.clear();
            ready.push_back(r);
            cv_work.notify_all();
        }
    }

    void finish(Request *r)
    {
        lpmgpu_batch_member(batch, r->member, &r->info);
        if (r->info.state == 1)
        {
            r->result.resize((size_t)r->desc.n * 3);
            lpmgpu_read_state(r->h, r->result.data(), nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
        }
        lpmgpu_batch_remove(batch, r->member);
        lpmgpu_destroy(r->h);
        r->h = nullptr;
        std::lock_guard<std::mutex> lk(mu);
        used -= r->bytes;
        running--;
        running_volume -= r->counted;
        r->t_done = Clock::now();
        if (r->info.state == 1)
        {
            r->state = 2;
            done++;
            latencies.push_back(std::chrono::duration<double>(r->t_done - r->t_submit).count());
        }
        else
        {
            r->state = 3;
            r->status = r->info.status;
            failed++;
        }
        finished_epoch++;
        cv_done.notify_all();
        cv_admit.notify_all();
    }

    void work()
    {
        cudaSetDevice(device);
        std::vector<Request *> live;
        for (;;)
        {
            std::vector<Request *> add;
            int64_t sl = -1;
            int32_t nl = 0;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_work.wait(lk, [&] { return stop || !ready.empty() || !live.empty(); });
                if (stop)
                    break;
                // admitted requests join while the running stream volume has room (in admission
                // order; a later, smaller one may pass a larger one that does not fit yet)
                if (solo_request >= 0)
                {
                    solo_bytes = solo_request;
                    solo_request = -1;
                    lpmgpu_batch_set_solo_bytes(batch, solo_bytes);
                }
                std::vector<Request *> wait;
                int64_t vol = running_volume;
                for (Request *r : ready)
                {
                    const int64_t v = counted_volume(r);
                    if ((live.empty() && add.empty()) || vol + v <= volume_cap)
                    {
                        add.push_back(r);
                        vol += v;
                    }
                    else
                        wait.push_back(r);
                }
                ready.swap(wait);
                sl = slice;
                slice = -1;
                if (lanes > 0 && live.empty())
                {
                    nl = lanes;
                    lanes = 0;
                }
            }
            if (sl >= 0)
                lpmgpu_batch_set_slice(batch, sl);
            if (nl > 0)
                lpmgpu_batch_set_lanes(batch, nl);
            for (Request *r : add)
            {
                std::vector<lpmgpu_load_step> v;
                for (auto &s : r->steps)
                    v.push_back(s.view);
                int32_t mid = -1;
                const int32_t s =
                    r->fatigue ? lpmgpu_batch_add_fatigue(batch, r->h, v.data(), r->nstatic, v.data() + r->nstatic,
                                                          r->cycle_len, r->ncycles, r->dndt.data(), &mid)
                               : lpmgpu_batch_add(batch, r->h, v.data(), (int32_t)v.size(), &mid);
                std::lock_guard<std::mutex> lk(mu);
                if (s != LPMGPU_OK)
                {
                    lpmgpu_destroy(r->h);
                    r->h = nullptr;
                    used -= r->bytes;
                    r->state = 3;
                    r->status = s;
                    r->t_done = Clock::now();
                    failed++;
                    finished_epoch++;
                    cv_done.notify_all();
                    cv_admit.notify_all();
                    continue;
                }
                r->member = mid;
                r->state = 1;
                r->t_start = Clock::now();
                running++;
                r->counted = counted_volume(r);
                running_volume += r->counted;
                live.push_back(r);
            }
            if (live.empty())
                continue;
            int32_t still = 0;
            const int32_t s = lpmgpu_batch_round(batch, &still);
            {
                std::lock_guard<std::mutex> lk(mu);
                rounds++;
                if (s != LPMGPU_OK)
                    worker_status = s;
            }
            if (s != LPMGPU_OK)
            {
                // the batch cannot go on: fail what is running and start a fresh batch
                lpmgpu_batch_destroy(batch);
                batch = nullptr;
                for (Request *r : live)
                {
                    lpmgpu_destroy(r->h);
                    r->h = nullptr;
                    std::lock_guard<std::mutex> lk(mu);
                    used -= r->bytes;
                    running--;
                    running_volume -= r->counted;
                    r->state = 3;
                    r->status = s;
                    r->t_done = Clock::now();
                    failed++;
                    finished_epoch++;
                }
                live.clear();
                lpmgpu_batch_create(device, &batch);
                if (batch)
                    lpmgpu_batch_set_solo_bytes(batch, solo_bytes);
                cv_done.notify_all();
                cv_admit.notify_all();
                if (!batch)
                    break;
                continue;
            }
            std::vector<Request *> keep;
            for (Request *r : live)
            {
                lpmgpu_member_info mi{};
                lpmgpu_batch_member(batch, r->member, &mi);
                if (mi.state != 0)
                    finish(r);
                else
                    keep.push_back(r);
            }
            live.swap(keep);
        }
        for (Request *r : live)
        {
            lpmgpu_destroy(r->h);
            r->h = nullptr;
        }
    }
};

extern "C" {

int32_t lpmgpu_estimate_bytes(const lpmgpu_desc *d, int64_t *bytes)
{
    if (!d || !bytes || d->n <= 0)
        return LPMGPU_ERR_INVALID_ARG;
    *bytes = estimate_bytes(*d);
    return LPMGPU_OK;
}

int32_t lpmgpu_server_create(int32_t device, int64_t hbm_budget_bytes, lpmgpu_server **out)
{
    if (!out || hbm_budget_bytes <= 0)
        return LPMGPU_ERR_INVALID_ARG;
    *out = nullptr;
    lpmgpu_batch *b = nullptr;
    const int32_t s = lpmgpu_batch_create(device, &b);
    if (s != LPMGPU_OK)
        return s;
    auto *srv = new lpmgpu_server();
    srv->device = device;
    srv->budget = hbm_budget_bytes;
    if (const char *env = std::getenv("LPMGPU_SERVE_VOLUME_MB"))
        if (std::atoll(env) > 0)
            srv->volume_cap = std::atoll(env) << 20;
    srv->batch = b;
    srv->t0 = Clock::now();
    srv->admit_thread = std::thread([srv] { srv->admission(); });
    srv->work_thread = std::thread([srv] { srv->work(); });
    *out = srv;
    return LPMGPU_OK;
}

int32_t lpmgpu_server_destroy(lpmgpu_server *s)
{
    if (!s)
        return LPMGPU_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_admit.notify_all();
    s->cv_work.notify_all();
    s->cv_done.notify_all();
    s->admit_thread.join();
    s->work_thread.join();
    for (Request *r : s->ready)
        if (r->h)
            lpmgpu_destroy(r->h);
    if (s->batch)
        lpmgpu_batch_destroy(s->batch);
    delete s;
    return LPMGPU_OK;
}

int32_t lpmgpu_server_set_slice(lpmgpu_server *s, int64_t iterations)
{
    if (!s || iterations < 0)
        return LPMGPU_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    s->slice = iterations; // applied by the worker before its next round
    return LPMGPU_OK;
}

int32_t lpmgpu_server_set_lanes(lpmgpu_server *s, int32_t lanes)
{
    if (!s || lanes < 1)
        return LPMGPU_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    s->lanes = lanes; // applied by the worker once no request is running
    s->cv_work.notify_all();
    return LPMGPU_OK;
}

int32_t lpmgpu_server_set_solo_bytes(lpmgpu_server *s, int64_t bytes)
{
    if (!s || bytes < 0)
        return LPMGPU_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    s->solo_request = bytes; // applied by the worker before its next admissions
    s->cv_work.notify_all();
    return LPMGPU_OK;
}

struct FatigueSpec
{
    int32_t nstatic, cycle_len, ncycles;
    const double *dndt;
};

// The request: a deep copy of the problem description and its steps (all static, or for a
// fatigue request the static steps followed by the cycles' steps)
static int32_t submit_impl(lpmgpu_server *s, const lpmgpu_desc *d, const lpmgpu_load_step *steps, int32_t nsteps,
                           int64_t *id, const FatigueSpec *f)
{
    if (!s || !d || !d->xyz || d->n <= 0 || nsteps < 0 || (nsteps > 0 && !steps))
        return LPMGPU_ERR_INVALID_ARG;
    if (d->device != s->device)
    {
        lpm::set_last_error("the request names another device than the server's");
        return LPMGPU_ERR_INVALID_ARG;
    }
    auto r = std::make_unique<Request>();
    r->desc = *d;
    const size_t n = (size_t)d->n;
    r->xyz.assign(d->xyz, d->xyz + 3 * n);
    r->desc.xyz = r->xyz.data();
    if (d->type)
    {
        r->type.assign(d->type, d->type + n);
        r->desc.type = r->type.data();
    }
    if (d->bond_nb0 && d->bond_nb1 && d->bond_p2)
    {
        r->nb0.assign(d->bond_nb0, d->bond_nb0 + n);
        r->nb1.assign(d->bond_nb1, d->bond_nb1 + n);
        size_t nb = 0;
        for (size_t i = 0; i < n; ++i)
            nb += (size_t)std::max(0, d->bond_nb0[i]) + (size_t)std::max(0, d->bond_nb1[i]);
        r->p2.assign(d->bond_p2, d->bond_p2 + nb);
        r->desc.bond_nb0 = r->nb0.data();
        r->desc.bond_nb1 = r->nb1.data();
        r->desc.bond_p2 = r->p2.data();
        if (d->bond_kn)
        {
            r->kn.assign(d->bond_kn, d->bond_kn + nb);
            r->desc.bond_kn = r->kn.data();
        }
        if (d->bond_tv)
        {
            r->tv.assign(d->bond_tv, d->bond_tv + nb);
            r->desc.bond_tv = r->tv.data();
        }
        if (d->bond_damage)
        {
            r->bdmg.assign(d->bond_damage, d->bond_damage + nb);
            r->desc.bond_damage = r->bdmg.data();
        }
    }
    if (d->nonlocal_count && d->nonlocal_ids)
    {
        r->nl_count.assign(d->nonlocal_count, d->nonlocal_count + n);
        size_t nl = 0;
        for (size_t i = 0; i < n; ++i)
            nl += (size_t)std::max(0, d->nonlocal_count[i]);
        r->nl_ids.assign(d->nonlocal_ids, d->nonlocal_ids + nl);
        r->desc.nonlocal_count = r->nl_count.data();
        r->desc.nonlocal_ids = r->nl_ids.data();
    }
    for (int32_t k = 0; k < nsteps; ++k)
        r->steps.emplace_back(steps[k]);
    if (f)
    {
        r->fatigue = true;
        r->nstatic = f->nstatic;
        r->cycle_len = f->cycle_len;
        r->ncycles = f->ncycles;
        r->dndt.assign(f->dndt, f->dndt + f->ncycles);
        if (r->dndt.empty())
            r->dndt.push_back(0.0);
    }
    r->est_bytes = estimate_bytes(r->desc);
    r->t_submit = Clock::now();
    std::lock_guard<std::mutex> lk(s->mu);
    r->id = s->next_id++;
    if (id)
        *id = r->id;
    s->queue.push_back(r.get());
    s->reqs[r->id] = std::move(r);
    s->submitted++;
    s->cv_admit.notify_all();
    return LPMGPU_OK;
}

int32_t lpmgpu_server_submit(lpmgpu_server *s, const lpmgpu_desc *d, const lpmgpu_load_step *steps, int32_t nsteps,
                             int64_t *id)
{
    return submit_impl(s, d, steps, nsteps, id, nullptr);
}

int32_t lpmgpu_server_submit_fatigue(lpmgpu_server *s, const lpmgpu_desc *d, const lpmgpu_load_step *static_steps,
                                     int32_t nstatic, const lpmgpu_load_step *cycle_steps, int32_t cycle_len,
                                     int32_t ncycles, const double *dndt, int64_t *id)
{
    if (nstatic < 0 || cycle_len < 0 || ncycles < 0 || (nstatic > 0 && !static_steps) ||
        (ncycles > 0 && (cycle_len == 0 || !cycle_steps || !dndt)))
        return LPMGPU_ERR_INVALID_ARG;
    std::vector<lpmgpu_load_step> all(static_steps, static_steps + nstatic);
    all.insert(all.end(), cycle_steps, cycle_steps + (size_t)cycle_len * ncycles);
    const FatigueSpec f{nstatic, cycle_len, ncycles, dndt};
    return submit_impl(s, d, all.data(), (int32_t)all.size(), id, &f);
}

static void fill_info(const lpmgpu_server *s, const Request &r, lpmgpu_request_info *info)
{
    std::memset(info, 0, sizeof(*info));
    info->state = r.state;
    info->status = r.status;
    info->n = r.desc.n;
    info->steps_done = r.info.steps_done;
    info->nsteps = (int32_t)r.steps.size();
    info->total = r.info.total;
    info->dof_iters = r.info.dof_iters;
    info->device_bytes = r.bytes;
    info->t_submit = s->since(r.t_submit);
    info->t_start = r.state >= 1 && r.t_start.time_since_epoch().count() ? s->since(r.t_start) : -1.0;
    info->t_done = r.state >= 2 ? s->since(r.t_done) : -1.0;
}

int32_t lpmgpu_server_poll(lpmgpu_server *s, int64_t id, lpmgpu_request_info *info)
{
    if (!s || !info)
        return LPMGPU_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end())
        return LPMGPU_ERR_INVALID_ARG;
    fill_info(s, *it->second, info);
    return LPMGPU_OK;
}

int32_t lpmgpu_server_wait(lpmgpu_server *s, int64_t id, double timeout_s, lpmgpu_request_info *info)
{
    if (!s)
        return LPMGPU_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end())
        return LPMGPU_ERR_INVALID_ARG;
    Request *r = it->second.get();
    const bool fin = s->cv_done.wait_for(lk, std::chrono::duration<double>(std::max(0.0, timeout_s)),
                                         [&] { return r->state >= 2 || s->stop; });
    if (info)
        fill_info(s, *r, info);
    return fin && r->state >= 2 ? LPMGPU_OK : LPMGPU_ERR_NOT_READY;
}

int32_t lpmgpu_server_result(lpmgpu_server *s, int64_t id, double *xyz, int64_t cap)
{
    if (!s)
        return LPMGPU_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end())
        return LPMGPU_ERR_INVALID_ARG;
    Request &r = *it->second;
    if (r.state < 2)
        return LPMGPU_ERR_NOT_READY;
    if (r.state == 3)
    {
        const int32_t st = r.status != LPMGPU_OK ? r.status : LPMGPU_ERR_NEWTON;
        s->reqs.erase(it);
        return st;
    }
    if (xyz)
    {
        if (cap < (int64_t)r.result.size())
            return LPMGPU_ERR_INVALID_ARG;
        std::memcpy(xyz, r.result.data(), sizeof(double) * r.result.size());
    }
    s->reqs.erase(it);
    return LPMGPU_OK;
}

int32_t lpmgpu_server_get_stats(lpmgpu_server *s, lpmgpu_server_stats *st)
{
    if (!s || !st)
        return LPMGPU_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    std::memset(st, 0, sizeof(*st));
    st->submitted = s->submitted;
    st->queued = (int64_t)s->queue.size();
    st->running = s->running + (int64_t)s->ready.size();
    st->done = s->done;
    st->failed = s->failed;
    st->rounds = s->rounds;
    st->bytes_in_use = s->used;
    st->bytes_budget = s->budget;
    st->peak_bytes = s->peak;
    st->worker_status = s->worker_status;
    if (!s->latencies.empty())
    {
        std::vector<double> l = s->latencies;
        std::sort(l.begin(), l.end());
        auto pct = [&](double p) {
            const double x = p * (double)(l.size() - 1);
            const size_t i = (size_t)x;
            const double f = x - (double)i;
            return i + 1 < l.size() ? l[i] * (1 - f) + l[i + 1] * f : l[i];
        };
        st->latency_p50 = pct(0.50);
        st->latency_p99 = pct(0.99);
    }
    st->seconds = s->since(Clock::now());
    return LPMGPU_OK;
}

} // extern "C"
