// gp5cu_batch.cu - batched independent LHY droplet ground states (imaginary-time RK4).
//
// Solves are grouped by grid size; a group is one plan carrying nsolve solves, so every axis
// pass of the group is a single launch over all of its solves (per-solve box, coefficients,
// time step and normalisation come from the SolveParams array, per-solve sums from the
// per-solve reductions).  Between convergence checks the group replays a CUDA graph of
// check_every merged RK4 steps; at a check the pending normalisation is applied, H psi and the
// residual are reduced per solve, and converged solves are switched off (their tiles return
// at once in every later launch).
#include <cmath>
#include <map>
#include <string>
#include <vector>

#include "plan.hpp"

using namespace gp5;

struct BatchGroup {
    int n = 0;
    std::vector<int> idx;  // global indices of the solves in this group
    gp5cu_plan *plan = nullptr;
    gp5cu_functional *func = nullptr;
    gp5cu_stepper *st = nullptr;
    void *psi = nullptr;  // nsolve consecutive fields
    std::vector<DevScalars> ds_host;
};

struct gp5cu_batch {
    int prec = GP5_C128;
    int dev = 0;
    std::vector<gp5cu_solve_desc> solves;
    std::vector<BatchGroup> groups;
    std::vector<int> group_of, slot_of;
    long long launches = 0;
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

// active flags of the stepper's and the functional's parameter arrays
void set_active(BatchGroup &g, const std::vector<int> &active) {
    for (size_t q = 0; q < g.idx.size(); q++) {
        g.st->sp_host[q].active = active[q];
        g.func->sp_host[q].active = active[q];
    }
    upload_params(g.st->sp_host, &g.st->sp);
    upload_params(g.func->sp_host, &g.func->sp);
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

int gp5cu_batch_create(gp5cu_batch **out, int nsolves, const gp5cu_solve_desc *solves, int precision, int device) {
    GP5B_TRY
    require_b(out && solves, "NULL argument");
    *out = nullptr;
    require_b(nsolves >= 1, "at least one solve");
    require_b(precision == GP5_C128 || precision == GP5_C64, "precision must be GP5_C128 or GP5_C64");
    for (int i = 0; i < nsolves; i++) {
        const gp5cu_solve_desc &d = solves[i];
        require_b(d.n == 32 || d.n == 64 || d.n == 128 || d.n == 256 || d.n == 512,
                  "batched grids must be powers of two in [32, 512]");
        require_b(d.L > 0 && d.N > 0 && d.dt > 0, "L, N and dt must be positive");
        require_b(std::isfinite(d.c3) && std::isfinite(d.c4) && d.omega >= 0, "invalid coefficients");
    }
    gp5cu_batch *b = new gp5cu_batch();
    try {
        b->prec = precision;
        b->dev = device;
        b->solves.assign(solves, solves + nsolves);
        b->group_of.resize(nsolves);
        b->slot_of.resize(nsolves);
        std::map<int, int> gid;
        for (int i = 0; i < nsolves; i++) {
            auto it = gid.find(solves[i].n);
            if (it == gid.end()) {
                gid[solves[i].n] = (int)b->groups.size();
                b->groups.emplace_back();
                b->groups.back().n = solves[i].n;
                it = gid.find(solves[i].n);
            }
            BatchGroup &g = b->groups[it->second];
            b->group_of[i] = it->second;
            b->slot_of[i] = (int)g.idx.size();
            g.idx.push_back(i);
        }
        for (BatchGroup &g : b->groups) {
            const int k = (int)g.idx.size();
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
        }
    } catch (...) {
        gp5cu_batch_destroy(b);
        throw;
    }
    *out = b;
    GP5B_CATCH
}

int gp5cu_batch_destroy(gp5cu_batch *b) {
    if (!b) return GP5_OK;
    for (BatchGroup &g : b->groups) destroy_group(g);
    delete b;
    return GP5_OK;
}

int gp5cu_batch_set_state(gp5cu_batch *b, int solve, const double *host) {
    GP5B_TRY
    require_b(b && host, "NULL argument");
    require_b(solve >= 0 && solve < (int)b->solves.size(), "solve index out of range");
    BatchGroup &g = b->groups[b->group_of[solve]];
    gp5cu_plan *p = g.plan;
    check_cuda(cudaSetDevice(p->dev), "cudaSetDevice");
    char *dst = static_cast<char *>(g.psi) + (size_t)b->slot_of[solve] * p->field_bytes;
    const int rc = gp5cu_upload_c128(p, dst, host);
    if (rc != GP5_OK) return rc;
    GP5B_CATCH
}

int gp5cu_batch_get_state(gp5cu_batch *b, int solve, double *host) {
    GP5B_TRY
    require_b(b && host, "NULL argument");
    require_b(solve >= 0 && solve < (int)b->solves.size(), "solve index out of range");
    BatchGroup &g = b->groups[b->group_of[solve]];
    gp5cu_plan *p = g.plan;
    check_cuda(cudaSetDevice(p->dev), "cudaSetDevice");
    const char *src = static_cast<const char *>(g.psi) + (size_t)b->slot_of[solve] * p->field_bytes;
    const int rc = gp5cu_download_c128(p, src, host);
    if (rc != GP5_OK) return rc;
    GP5B_CATCH
}

int gp5cu_batch_solve(gp5cu_batch *b, double tol, int check_every, int max_steps, gp5cu_solve_result *results) {
    GP5B_TRY
    require_b(b && results, "NULL argument");
    require_b(tol > 0 && check_every >= 1 && max_steps >= 0, "invalid tolerance or step counts");
    const int ns = (int)b->solves.size();
    std::vector<int> steps(ns, 0), done(ns, 0);
    b->launches = 0;
    for (BatchGroup &g : b->groups) {
        check_cuda(cudaSetDevice(g.plan->dev), "cudaSetDevice");
        set_active(g, std::vector<int>(g.idx.size(), 1));
        if (!g.st->exec || g.st->graph_field != g.psi || g.st->graph_steps != check_every)
            build_graph(g.st, g.psi, true, check_every);
    }
    // check 0 looks at the initial states; every later check advances check_every steps first
    for (int check = 0;; check++) {
        bool any = false;
        for (BatchGroup &g : b->groups) {
            gp5cu_plan *p = g.plan;
            gp5cu_stepper *st = g.st;
            bool active = false;
            for (int i : g.idx) active = active || !done[i];
            if (!active) continue;
            any = true;
            dispatch_b(b->prec, [&](auto r) {
                using Real = decltype(r);
                if (check > 0) {
                    set_scalars(p->stream, st->ds, p->nsolve);
                    Launch<Real>::prologue(st, g.psi);
                    check_cuda(cudaGraphLaunch(st->exec, p->stream), "cudaGraphLaunch");
                    Launch<Real>::scale(p, g.psi, -1, st->ds, true);  // pending normalisation
                    b->launches += 3 + (long long)check_every * st->launches_per_step;
                }
                set_scalars(p->stream, p->ds, p->nsolve);
                Launch<Real>::apply_h(g.func, g.psi, p->work, true);
                Launch<Real>::residual(p, g.psi, p->work, p->ds, g.func->sp);
                b->launches += 7;
            });
            check_cuda(cudaMemcpyAsync(g.ds_host.data(), p->ds, sizeof(DevScalars) * g.idx.size(),
                                       cudaMemcpyDeviceToHost, p->stream),
                       "read batch sums");
        }
        if (!any) break;
        bool all_done = true;
        for (BatchGroup &g : b->groups) {
            check_cuda(cudaStreamSynchronize(g.plan->stream), "sync");
            std::vector<int> act(g.idx.size(), 1);
            for (size_t q = 0; q < g.idx.size(); q++) {
                const int i = g.idx[q];
                if (done[i]) {
                    act[q] = 0;
                    continue;
                }
                if (check > 0) steps[i] += check_every;
                const DevScalars &d = g.ds_host[q];
                const double dV = g.plan->sp_host[q].dV;
                gp5cu_solve_result &R = results[i];
                R.steps = steps[i];
                R.norm = d.sums[0] * dV;
                R.energy = (d.sums[1] + d.sums[2] + d.sums[3]) * dV;
                R.mu = d.sums[4] / d.sums[0];
                R.residual = std::sqrt(d.sums[5] / d.sums[0]);
                R.converged = (R.residual <= tol) ? 1 : 0;
                if (!std::isfinite(R.residual)) fail(GP5_ERR_NONFINITE, "solve " + std::to_string(i) + " diverged");
                if (R.converged || steps[i] >= max_steps) {
                    done[i] = 1;
                    act[q] = 0;
                } else {
                    all_done = false;
                }
            }
            set_active(g, act);
        }
        if (all_done) break;
    }
    GP5B_CATCH
}

long long gp5cu_batch_launches(const gp5cu_batch *b) { return b ? b->launches : 0; }

}  // extern "C"
