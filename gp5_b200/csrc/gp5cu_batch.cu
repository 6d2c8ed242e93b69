// gp5cu_batch.cu - batched independent LHY droplet ground states (imaginary-time RK4).
//
// Solves are grouped by grid size; a group is one plan carrying its solves in consecutive
// slots, so every axis pass of the group is a single launch over all of its live solves
// (per-solve box, coefficients, time step and normalisation come from the SolveParams array,
// per-solve sums from the per-solve reductions).  Between convergence checks the group
// replays CUDA graphs of merged RK4 steps; at a check the pending normalisation is applied,
// H psi and the residual are reduced per solve, and solves that are finished leave the launch
// grid: the live solves are packed into the first slots (device-to-device copies of their
// states and a permutation of the parameter arrays) and the plan's solve count shrinks to
// them, so a long tail of slow solves runs only its own tiles.
//
// complex64 batches run in two phases: every solve advances with complex64 state and
// transforms (FP64 reductions) until its residual reaches GP5_BATCH_SWITCH_RESIDUAL or stops
// falling near the complex64 floor; then all states are converted to complex128 and a
// complex128 group takes every solve to the requested tolerance.
#include <algorithm>
#include <cmath>
#include <map>
#include <string>
#include <vector>

#include "plan.hpp"

using namespace gp5;

struct BatchGroup {
    int n = 0;
    int dev = 0;
    int prec = GP5_C128;
    std::vector<int> idx;  // slot -> global solve index
    int live = 0;          // slots [0, live) are in the launches (plan->nsolve == live when > 0)
    gp5cu_plan *plan = nullptr;
    gp5cu_functional *func = nullptr;
    gp5cu_stepper *st = nullptr;
    void *psi = nullptr;  // idx.size() consecutive fields
    std::vector<DevScalars> ds_host;
    std::vector<DevScalars> st_host;  // the stepper's scalars (status of the bounded waits)
    // graph of `pexec_iters` preconditioned iterations over `pexec_live` live solves
    cudaGraphExec_t pexec = nullptr;
    int pexec_iters = 0, pexec_live = 0;
};

struct gp5cu_batch {
    int prec = GP5_C128;
    std::vector<int> devices;     // devices the solves are spread over
    std::vector<int> device_of;   // per solve: its device ordinal
    std::vector<gp5cu_solve_desc> solves;
    // groups[0]: the batch precision; groups[1]: the complex128 groups of a complex64 batch
    std::vector<BatchGroup> groups[2];
    std::vector<int> group_of[2], slot_of[2];
    std::vector<char> in_c128;  // complex64 batch: the current state is the complex128 group's
    long long launches = 0;
    int method = GP5_BATCH_RK4;  // gp5cu_batch_set_method
    double theta = 0.5;
};

namespace {

void require_b(bool c, const std::string &m) {
    if (!c) fail(GP5_ERR_ARG, m);
}

void destroy_group(BatchGroup &g) {
    if (g.plan) {
        cudaSetDevice(g.plan->dev);
        cudaStreamSynchronize(g.plan->stream);
    }
    if (g.pexec) cudaGraphExecDestroy(g.pexec);
    g.pexec = nullptr;
    if (g.st) gp5cu_stepper_destroy(g.st);
    if (g.func) gp5cu_functional_destroy(g.func);
    if (g.psi) cudaFree(g.psi);
    if (g.plan) gp5cu_plan_destroy(g.plan);
    g.st = nullptr;
    g.func = nullptr;
    g.psi = nullptr;
    g.plan = nullptr;
}

template <class F> void dispatch_b(int prec, F &&f) {
    if (prec == GP5_C128) f((double)0);
    else f((float)0);
}

// Steps per captured graph: the largest divisor of check_every not above 100 (a graph of a few
// hundred launches captures in milliseconds when the live set changes).
int graph_chunk(int check_every) {
    for (int k = std::min(check_every, 100); k >= 1; k--)
        if (check_every % k == 0) return k;
    return 1;
}

// Builds one group (plan, LHY functional, renormalised imaginary-time RK4 stepper, states) for
// the given global solve indices, all of grid size n.
void make_group(BatchGroup &g, const std::vector<gp5cu_solve_desc> &solves, int precision) {
    const int device = g.dev;
    const int k = (int)g.idx.size();
    g.prec = precision;
    std::vector<double> lv(3 * k), rv(3 * k);
    std::vector<const double *> lp(k), rp(k);
    bool trap = false;
    for (int q = 0; q < k; q++) {
        const gp5cu_solve_desc &d = solves[g.idx[q]];
        for (int a = 0; a < 3; a++) {
            lv[3 * q + a] = -d.L / 2;
            rv[3 * q + a] = d.L / 2;
        }
        lp[q] = &lv[3 * q];
        rp[q] = &rv[3 * q];
        trap = trap || d.omega > 0;
    }
    const int shape[3] = {g.n, g.n, g.n};
    g.plan = create_plan(shape, lp.data(), rp.data(), k, 1, precision, device);
    gp5cu_functional_desc fd;
    gp5cu_functional_desc_init(&fd);
    fd.kind = GP5_FUNC_LHY;
    if (trap) fd.potential = GP5_POT_HARMONIC;
    int rc = gp5cu_functional_create(g.plan, &fd, &g.func);
    if (rc != GP5_OK) fail(rc, gp5cu_last_error());
    for (int q = 0; q < k; q++) {
        const gp5cu_solve_desc &d = solves[g.idx[q]];
        SolveParams &S = g.func->sp_host[q];
        S.c3 = d.c3;
        S.c4 = d.c4;
        for (int a = 0; a < 3; a++) S.om2[0][a] = d.omega * d.omega;
    }
    upload_params(g.func->sp_host, &g.func->sp);
    rc = gp5cu_stepper_create(g.func, GP5_STEP_RK4, solves[g.idx[0]].dt, 1, &g.st);
    if (rc != GP5_OK) fail(rc, gp5cu_last_error());
    g.st->renorm = true;
    for (int q = 0; q < k; q++) {
        const gp5cu_solve_desc &d = solves[g.idx[q]];
        SolveParams &S = g.st->sp_host[q];
        S = g.func->sp_host[q];
        S.tre = d.dt;  // imaginary time: tau = (dt, 0)
        S.tim = 0.0;
        S.Nt[0] = d.N;
        S.Nt[1] = 0.0;
    }
    upload_params(g.st->sp_host, &g.st->sp);
    check_cuda(cudaMalloc(&g.psi, g.plan->field_bytes * k), "cudaMalloc batch states");
    check_cuda(cudaMemset(g.psi, 0, g.plan->field_bytes * k), "memset batch states");
    g.ds_host.resize(k);
    g.st_host.resize(k);
    g.live = k;
}

// Puts the first `live` slots into the launches: active flags, the plan's solve count and the
// point-wise grid; the stepper's graph is dropped when the count changes (rebuilt lazily).
void set_live(BatchGroup &g, int live) {
    const int cap = (int)g.idx.size();
    for (int q = 0; q < cap; q++) {
        g.st->sp_host[q].active = q < live;
        g.func->sp_host[q].active = q < live;
    }
    upload_params(g.st->sp_host, &g.st->sp);
    upload_params(g.func->sp_host, &g.func->sp);
    g.live = live;
    if (live > 0 && g.plan->nsolve != live) {
        gp5cu_plan *p = g.plan;
        p->nsolve = live;
        // point-wise blocks per solve, within the partial-sum slots each solve owns
        p->pw_bps = (int)std::min<long long>(p->max_blocks, std::max(1, p->pw_blocks / live));
        drop_graph(g.st);
    }
}

// Packs the slots whose keep flag is set (among the live ones) to the front, in their current
// order, followed by the other slots; their states move with them (through the work field,
// which holds as many fields as the group has slots) and so do the parameter arrays.
// slot_of receives every moved solve's new slot.  Then only the kept slots stay live.
void repack(BatchGroup &g, const std::vector<char> &keep, std::vector<int> &slot_of) {
    const int cap = (int)g.idx.size();
    std::vector<int> order;
    for (int q = 0; q < g.live; q++)
        if (keep[q]) order.push_back(q);
    const int live = (int)order.size();
    for (int q = 0; q < cap; q++)
        if (q >= g.live || !keep[q]) order.push_back(q);
    bool moved = false;
    for (int j = 0; j < cap; j++) moved = moved || order[j] != j;
    gp5cu_plan *p = g.plan;
    if (moved) {
        const size_t fb = p->field_bytes;
        char *W = static_cast<char *>(p->work), *S = static_cast<char *>(g.psi);
        for (int j = 0; j < cap; j++)
            if (order[j] != j)
                check_cuda(cudaMemcpyAsync(W + j * fb, S + order[j] * fb, fb, cudaMemcpyDeviceToDevice, p->stream),
                           "pack batch states");
        for (int j = 0; j < cap; j++)
            if (order[j] != j)
                check_cuda(cudaMemcpyAsync(S + j * fb, W + j * fb, fb, cudaMemcpyDeviceToDevice, p->stream),
                           "pack batch states");
        auto permute = [&](auto &v) {
            auto old = v;
            for (int j = 0; j < cap; j++) v[j] = old[order[j]];
        };
        permute(g.idx);
        permute(p->sp_host);
        permute(g.func->sp_host);
        permute(g.st->sp_host);
        check_cuda(cudaMemcpyAsync(p->sp_lap, p->sp_host.data(), sizeof(SolveParams) * cap, cudaMemcpyHostToDevice,
                                   p->stream),
                   "upload params");
        check_cuda(cudaStreamSynchronize(p->stream), "sync");
        for (int j = 0; j < cap; j++) slot_of[g.idx[j]] = j;
    }
    set_live(g, live);
}

// Converts the state of solve i between its complex64 slot (groups[0]) and its complex128
// slot (groups[1]), in the direction `to128`.
void convert_state(gp5cu_batch *b, int i, bool to128) {
    BatchGroup &g32 = b->groups[0][b->group_of[0][i]];
    BatchGroup &g64 = b->groups[1][b->group_of[1][i]];
    void *s32 = static_cast<char *>(g32.psi) + (size_t)b->slot_of[0][i] * g32.plan->field_bytes;
    void *s64 = static_cast<char *>(g64.psi) + (size_t)b->slot_of[1][i] * g64.plan->field_bytes;
    const long long n = g32.plan->nsites;
    check_cuda(cudaSetDevice(g32.plan->dev), "cudaSetDevice");
    if (to128) Launch<float>::convert(g32.plan, nullptr, nullptr, s32, static_cast<double *>(s64), n);
    else Launch<float>::convert(g32.plan, static_cast<const double *>(s64), s32, nullptr, nullptr, n);
    b->launches += 1;
}

// Queues `iters` preconditioned iterations of every live solve of group g on its plan stream.
void queue_precond(BatchGroup &g, int iters, double theta) {
    dispatch_b(g.prec, [&](auto r) {
        using Real = decltype(r);
        for (int k = 0; k < iters; k++) Launch<Real>::precond_iter(g.func, g.st->sp, g.psi, g.st->Ka, theta);
    });
}

// Captures `iters` preconditioned iterations of group g into g.pexec (after a configuring
// pass that launches nothing, as for the step graphs).
void build_precond_graph(BatchGroup &g, int iters, double theta) {
    gp5cu_plan *p = g.plan;
    if (g.pexec) cudaGraphExecDestroy(g.pexec);
    g.pexec = nullptr;
    p->dry = true;
    try {
        queue_precond(g, 1, theta);
    } catch (...) {
        p->dry = false;
        throw;
    }
    p->dry = false;
    cudaGraph_t gr = nullptr;
    check_cuda(cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    try {
        queue_precond(g, iters, theta);
    } catch (...) {
        cudaStreamEndCapture(p->stream, &gr);
        if (gr) cudaGraphDestroy(gr);
        throw;
    }
    check_cuda(cudaStreamEndCapture(p->stream, &gr), "end capture");
    const cudaError_t e = cudaGraphInstantiate(&g.pexec, gr, 0);
    cudaGraphDestroy(gr);
    check_cuda(e, "cudaGraphInstantiate");
    g.pexec_iters = iters;
    g.pexec_live = g.live;
}

// Imaginary-time RK4 (or, with GP5_BATCH_PRECOND, the preconditioned iteration) of every
// solve of `groups` until done(i, residual, residual at the
// previous check, steps taken in this phase) says so or the phase's step budget runs out;
// results[i] holds the last check's observables.  Returns the steps of this phase per solve.
template <class Done>
std::vector<int> run_phase(gp5cu_batch *b, int set, int check_every, const std::vector<int> &budget,
                           gp5cu_solve_result *results, Done done_fn) {
    std::vector<BatchGroup> &groups = b->groups[set];
    const int ns = (int)b->solves.size();
    std::vector<int> steps(ns, 0);
    std::vector<double> prev(ns, INFINITY);
    const int chunk = graph_chunk(check_every);
    for (BatchGroup &g : groups) {
        check_cuda(cudaSetDevice(g.plan->dev), "cudaSetDevice");
        set_live(g, (int)g.idx.size());
    }
    // check 0 looks at the current states; every later check advances check_every steps first
    for (int check = 0;; check++) {
        bool any = false;
        for (BatchGroup &g : groups) {
            if (g.live == 0) continue;
            any = true;
            gp5cu_plan *p = g.plan;
            gp5cu_stepper *st = g.st;
            check_cuda(cudaSetDevice(p->dev), "cudaSetDevice");
            dispatch_b(g.prec, [&](auto r) {
                using Real = decltype(r);
                if (check > 0 && b->method == GP5_BATCH_PRECOND) {
                    // the check's reset scalars hold sigma = 1: the iterations read psi as stored
                    if (!g.pexec || g.pexec_live != g.live || g.pexec_iters != chunk)
                        build_precond_graph(g, chunk, b->theta);
                    for (int k = 0; k < check_every; k += chunk)
                        check_cuda(cudaGraphLaunch(g.pexec, p->stream), "cudaGraphLaunch");
                    b->launches += (long long)check_every * Launch<Real>::kPrecondLaunches;
                } else if (check > 0) {
                    if (!st->exec || st->graph_field != g.psi || st->graph_steps != chunk)
                        build_graph(st, g.psi, true, chunk);
                    set_scalars(p->stream, st->ds, p->nsolve);
                    Launch<Real>::prologue(st, g.psi);
                    for (int k = 0; k < check_every; k += chunk)
                        check_cuda(cudaGraphLaunch(st->exec, p->stream), "cudaGraphLaunch");
                    Launch<Real>::scale(p, g.psi, -1, st->ds, true);  // pending normalisation
                    b->launches += 3 + (long long)check_every * st->launches_per_step;
                    check_cuda(cudaMemcpyAsync(g.st_host.data(), st->ds, sizeof(DevScalars) * g.live,
                                               cudaMemcpyDeviceToHost, p->stream),
                               "read batch step status");
                }
                set_scalars(p->stream, p->ds, p->nsolve);
                Launch<Real>::apply_h(g.func, g.psi, p->work, true);
                Launch<Real>::residual(p, g.psi, p->work, p->ds, g.func->sp);
                b->launches += 7;
            });
            check_cuda(cudaMemcpyAsync(g.ds_host.data(), p->ds, sizeof(DevScalars) * g.live, cudaMemcpyDeviceToHost,
                                       p->stream),
                       "read batch sums");
        }
        if (!any) break;
        bool any_live = false;
        for (BatchGroup &g : groups) {
            if (g.live == 0) continue;
            check_cuda(cudaSetDevice(g.plan->dev), "cudaSetDevice");
            check_cuda(cudaStreamSynchronize(g.plan->stream), "sync");
            std::vector<char> keep(g.live, 1);
            int kept = 0;
            for (int q = 0; q < g.live; q++) {
                const int i = g.idx[q];
                if (check > 0 && b->method == GP5_BATCH_RK4 && (g.st_host[q].status & DS_TIMEOUT))
                    fail(GP5_ERR_TIMEOUT, "a bounded device wait ran out (solve " + std::to_string(i) + ")");
                if (check > 0) steps[i] += check_every;
                const DevScalars &d = g.ds_host[q];
                const double dV = g.plan->sp_host[q].dV;
                gp5cu_solve_result &R = results[i];
                R.norm = d.sums[0] * dV;
                R.energy = (d.sums[1] + d.sums[2] + d.sums[3]) * dV;
                R.mu = d.sums[4] / d.sums[0];
                R.residual = std::sqrt(d.sums[5] / d.sums[0]);
                if (!std::isfinite(R.residual)) fail(GP5_ERR_NONFINITE, "solve " + std::to_string(i) + " diverged");
                if (done_fn(i, R.residual, prev[i]) || steps[i] >= budget[i]) keep[q] = 0;
                else kept++;
                prev[i] = R.residual;
            }
            if (kept != g.live) repack(g, keep, b->slot_of[set]);
            any_live = any_live || g.live > 0;
        }
        if (!any_live) break;
    }
    return steps;
}

// Groups the solves by (device, grid size) into b->groups[set] (one plan per pair).
void build_groups(gp5cu_batch *b, int set, int precision) {
    const int ns = (int)b->solves.size();
    b->group_of[set].assign(ns, 0);
    b->slot_of[set].assign(ns, 0);
    std::map<std::pair<int, int>, int> gid;
    for (int i = 0; i < ns; i++) {
        const std::pair<int, int> key(b->device_of[i], b->solves[i].n);
        auto it = gid.find(key);
        if (it == gid.end()) {
            it = gid.emplace(key, (int)b->groups[set].size()).first;
            b->groups[set].emplace_back();
            b->groups[set].back().n = key.second;
            b->groups[set].back().dev = key.first;
        }
        BatchGroup &g = b->groups[set][it->second];
        b->group_of[set][i] = it->second;
        b->slot_of[set][i] = (int)g.idx.size();
        g.idx.push_back(i);
    }
    for (BatchGroup &g : b->groups[set]) make_group(g, b->solves, precision);
}

}  // namespace

#define GP5B_TRY try {
#define GP5B_CATCH                              \
    }                                           \
    catch (const Gp5Error &e) {                 \
        set_last_error(e.msg);                  \
        return e.status;                        \
    }                                           \
    catch (const std::exception &e) {           \
        set_last_error(e.what());               \
        return GP5_ERR_ARG;                     \
    }                                           \
    return GP5_OK;

extern "C" {

int gp5cu_batch_assign_devices(int nsolves, const gp5cu_solve_desc *solves, int ndevices, int *device_index) {
    GP5B_TRY
    require_b(solves && device_index, "NULL argument");
    require_b(nsolves >= 1 && ndevices >= 1, "at least one solve and one device");
    for (int i = 0; i < nsolves; i++)
        require_b(solves[i].n >= 1 && solves[i].n <= 4096, "grid size out of range");
    // longest-processing-time-first: solves by decreasing sites (ties: lower index first),
    // each to the device with the fewest sites so far (ties: lower device index)
    std::vector<int> order(nsolves);
    for (int i = 0; i < nsolves; i++) order[i] = i;
    auto sites = [&](int i) { return (double)solves[i].n * solves[i].n * solves[i].n; };
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return sites(a) > sites(c); });
    std::vector<double> load(ndevices, 0.0);
    for (int i : order) {
        int best = 0;
        for (int d = 1; d < ndevices; d++)
            if (load[d] < load[best]) best = d;
        device_index[i] = best;
        load[best] += sites(i);
    }
    GP5B_CATCH
}

int gp5cu_batch_create_devices(gp5cu_batch **out, int nsolves, const gp5cu_solve_desc *solves, int precision,
                               int ndevices, const int *devices) {
    GP5B_TRY
    require_b(out && solves && devices, "NULL argument");
    *out = nullptr;
    require_b(nsolves >= 1, "at least one solve");
    require_b(ndevices >= 1 && ndevices <= 64, "between 1 and 64 devices");
    require_b(precision == GP5_C128 || precision == GP5_C64, "precision must be GP5_C128 or GP5_C64");
    for (int i = 0; i < nsolves; i++) {
        const gp5cu_solve_desc &d = solves[i];
        require_b(d.n == 32 || d.n == 64 || d.n == 128 || d.n == 256 || d.n == 512,
                  "batched grids must be powers of two in [32, 512]");
        require_b(d.L > 0 && d.N > 0 && d.dt > 0, "L, N and dt must be positive");
        require_b(std::isfinite(d.c3) && std::isfinite(d.c4) && d.omega >= 0, "invalid coefficients");
    }
    int ndev = 0;
    check_cuda(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
    for (int k = 0; k < ndevices; k++) {
        require_b(devices[k] >= 0 && devices[k] < ndev, "device ordinal out of range");
        for (int j = 0; j < k; j++) require_b(devices[j] != devices[k], "a device is listed twice");
    }
    gp5cu_batch *b = new gp5cu_batch();
    try {
        b->prec = precision;
        b->devices.assign(devices, devices + ndevices);
        b->solves.assign(solves, solves + nsolves);
        b->in_c128.assign(nsolves, 0);
        std::vector<int> di(nsolves);
        const int rc = gp5cu_batch_assign_devices(nsolves, solves, ndevices, di.data());
        if (rc != GP5_OK) fail(rc, gp5cu_last_error());
        b->device_of.resize(nsolves);
        for (int i = 0; i < nsolves; i++) b->device_of[i] = devices[di[i]];
        build_groups(b, 0, precision);
    } catch (...) {
        gp5cu_batch_destroy(b);
        throw;
    }
    *out = b;
    GP5B_CATCH
}

int gp5cu_batch_create(gp5cu_batch **out, int nsolves, const gp5cu_solve_desc *solves, int precision, int device) {
    return gp5cu_batch_create_devices(out, nsolves, solves, precision, 1, &device);
}

int gp5cu_batch_device(const gp5cu_batch *b, int solve) {
    if (!b || solve < 0 || solve >= (int)b->solves.size()) return -1;
    return b->device_of[solve];
}

int gp5cu_batch_destroy(gp5cu_batch *b) {
    if (!b) return GP5_OK;
    for (auto &set : b->groups)
        for (BatchGroup &g : set) destroy_group(g);
    delete b;
    return GP5_OK;
}

int gp5cu_batch_set_state(gp5cu_batch *b, int solve, const double *host) {
    GP5B_TRY
    require_b(b && host, "NULL argument");
    require_b(solve >= 0 && solve < (int)b->solves.size(), "solve index out of range");
    BatchGroup &g = b->groups[0][b->group_of[0][solve]];
    gp5cu_plan *p = g.plan;
    check_cuda(cudaSetDevice(p->dev), "cudaSetDevice");
    char *dst = static_cast<char *>(g.psi) + (size_t)b->slot_of[0][solve] * p->field_bytes;
    const int rc = gp5cu_upload_c128(p, dst, host);
    if (rc != GP5_OK) return rc;
    b->in_c128[solve] = 0;
    GP5B_CATCH
}

int gp5cu_batch_get_state(gp5cu_batch *b, int solve, double *host) {
    GP5B_TRY
    require_b(b && host, "NULL argument");
    require_b(solve >= 0 && solve < (int)b->solves.size(), "solve index out of range");
    const int set = b->in_c128[solve] ? 1 : 0;
    BatchGroup &g = b->groups[set][b->group_of[set][solve]];
    gp5cu_plan *p = g.plan;
    check_cuda(cudaSetDevice(p->dev), "cudaSetDevice");
    const char *src = static_cast<const char *>(g.psi) + (size_t)b->slot_of[set][solve] * p->field_bytes;
    const int rc = gp5cu_download_c128(p, src, host);
    if (rc != GP5_OK) return rc;
    GP5B_CATCH
}

int gp5cu_batch_solve(gp5cu_batch *b, double tol, int check_every, int max_steps, gp5cu_solve_result *results) {
    GP5B_TRY
    require_b(b && results, "NULL argument");
    require_b(tol > 0 && check_every >= 1 && max_steps >= 0, "invalid tolerance or step counts");
    const int ns = (int)b->solves.size();
    b->launches = 0;
    for (int i = 0; i < ns; i++) results[i] = gp5cu_solve_result{};
    if (b->prec == GP5_C128) {
        const std::vector<int> steps = run_phase(b, 0, check_every, std::vector<int>(ns, max_steps), results,
                                                 [&](int, double r, double) { return r <= tol; });
        for (int i = 0; i < ns; i++) {
            results[i].steps = steps[i];
            results[i].converged = results[i].residual <= tol;
        }
        return GP5_OK;
    }
    // complex64 batch: a state left in complex128 by an earlier call continues from there
    for (int i = 0; i < ns; i++)
        if (b->in_c128[i]) convert_state(b, i, false);
    for (BatchGroup &g : b->groups[0]) {
        check_cuda(cudaSetDevice(g.plan->dev), "cudaSetDevice");
        check_cuda(cudaStreamSynchronize(g.plan->stream), "sync");
    }
    for (int i = 0; i < ns; i++) b->in_c128[i] = 0;
    // phase 1, complex64: until the switch residual, or until the residual stops falling (it
    // has reached the complex64 floor)
    const double sw = std::max(tol, (double)GP5_BATCH_SWITCH_RESIDUAL);
    const std::vector<int> s32 = run_phase(b, 0, check_every, std::vector<int>(ns, max_steps), results,
                                           [&](int, double r, double rprev) {
                                               return r <= sw || (r < 1e-3 && r > 0.7 * rprev);
                                           });
    // phase 2, complex128, from the converted states
    if (b->groups[1].empty()) build_groups(b, 1, GP5_C128);
    for (int i = 0; i < ns; i++) convert_state(b, i, true);
    for (BatchGroup &g : b->groups[0]) {
        check_cuda(cudaSetDevice(g.plan->dev), "cudaSetDevice");
        check_cuda(cudaStreamSynchronize(g.plan->stream), "sync");
    }
    for (int i = 0; i < ns; i++) b->in_c128[i] = 1;
    std::vector<int> budget(ns);
    for (int i = 0; i < ns; i++) budget[i] = std::max(0, max_steps - s32[i]);
    const std::vector<int> s64 = run_phase(b, 1, check_every, budget, results,
                                           [&](int, double r, double) { return r <= tol; });
    for (int i = 0; i < ns; i++) {
        results[i].steps = s32[i] + s64[i];
        results[i].steps_c64 = s32[i];
        results[i].converged = results[i].residual <= tol;
    }
    GP5B_CATCH
}

int gp5cu_batch_set_method(gp5cu_batch *b, int method, double theta) {
    GP5B_TRY
    require_b(b != nullptr, "NULL argument");
    require_b(method == GP5_BATCH_RK4 || method == GP5_BATCH_PRECOND, "method must be GP5_BATCH_RK4 or GP5_BATCH_PRECOND");
    require_b(theta > 0 && theta <= 1, "theta must be in (0, 1]");
    if (method != b->method || theta != b->theta)
        for (auto &set : b->groups)
            for (BatchGroup &g : set) {
                if (g.pexec) {
                    check_cuda(cudaSetDevice(g.plan->dev), "cudaSetDevice");
                    cudaGraphExecDestroy(g.pexec);
                }
                g.pexec = nullptr;
            }
    b->method = method;
    b->theta = theta;
    GP5B_CATCH
}

long long gp5cu_batch_launches(const gp5cu_batch *b) { return b ? b->launches : 0; }

}  // extern "C"
