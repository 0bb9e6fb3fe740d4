// tmx_serve.cpp -- the request loop of the served form (tmx_serve and
// tmx_serve_with in include/tmx.h): continuous batching of T-mixer solves over
// an engine given as callbacks; tmx_serve binds it to a tmx_batch and the
// wall clock.
//
// Policy
//   - admission in arrival order: the next request is admitted once it has
//     arrived, every earlier one has been admitted (or rejected as larger than
//     the whole budget) and the engine can place it (the engine answers
//     TMX_E_NOMEM while its free arena is too small);
//   - all admitted mixers advance together, check_every steps at a time; the
//     last of those steps writes the macroscopic fields and the outlet mixing
//     index of every mixer is read;
//   - a mixer is retired when each species' outlet index is defined (the
//     species have reached the outlet) and moved by less than tol over its
//     last window steps, or when it reaches max_steps; its range
//     goes back to the engine and the next waiting request fills it before
//     the next chunk of steps;
//   - a mixer the engine reports as non-finite (optional health callback)
//     is retired at once with status TMX_E_NONFINITE;
//   - a request the engine cannot take at all (its footprint or add callback
//     fails with anything but TMX_E_NOMEM: an invalid case, a precision
//     other than the batch's) is finished at once with that error code as
//     its status, and the loop goes on with the others;
//   - an error of step, outlet_im, health or remove ends the loop with that
//     code, after every admitted mixer has been removed from the engine;
//   - with no mixer admitted, the loop idles until the next arrival.
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <deque>
#include <numeric>
#include <thread>
#include <vector>

#include "../../include/tmx.h"

namespace tmx_host {
int fail(int code, const char* fmt, ...);
}
using tmx_host::fail;

namespace {

struct Active {
    int req;
    int slot;
    long long steps = 0;
    std::deque<std::array<double, 3>> history;  // outlet index at the last checks, newest last
};

double nearest_rank(std::vector<double> v, double p)
{
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double r = std::ceil(p * (double)v.size());
    const size_t i = (size_t)std::max(1.0, r) - 1;
    return v[std::min(i, v.size() - 1)];
}

}  // namespace

extern "C" {

int tmx_serve_with(const tmx_serve_ops* ops, const tmx_request* reqs, int n, const tmx_serve_opts* opts,
                   tmx_served* out, double summary[8])
{
    if (!ops || !opts || (n > 0 && (!reqs || !out))) return fail(TMX_E_INVALID, "null argument");
    if (!ops->footprint || !ops->capacity || !ops->add || !ops->remove || !ops->step || !ops->outlet_im ||
        !ops->now || !ops->wait_until)
        return fail(TMX_E_INVALID, "tmx_serve_with: every callback is required");
    const int every = opts->check_every;
    if (every <= 0) return fail(TMX_E_INVALID, "check_every must be positive");
    for (int r = 0; r < n; r++) {
        const tmx_request& q = reqs[r];
        if (q.max_steps <= 0 || q.window <= 0 || q.window % every)
            return fail(TMX_E_INVALID, "request %d: max_steps > 0 and window a positive multiple of check_every (%d)",
                        r, every);
        if (!(q.arrival >= 0) || !(q.tol >= 0)) return fail(TMX_E_INVALID, "request %d: bad arrival or tol", r);
    }
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return reqs[a].arrival < reqs[b].arrival; });
    for (int r = 0; r < n; r++) {
        out[r] = tmx_served{};
        out[r].status = -100;  // not served yet
        out[r].slot = -1;
    }
    const long long cap = ops->capacity(ops->ctx);
    std::vector<Active> active;
    // a fatal engine error: give every admitted range back, then report it
    auto abort_with = [&](int code) {
        for (const Active& a : active) ops->remove(ops->ctx, a.slot);
        active.clear();
        return code;
    };
    size_t next = 0;  // next request (in arrival order) not yet admitted
    int done = 0;
    long long lups = 0, checks = 0;
    int most = 0;
    double area = 0.0, last_t = ops->now(ops->ctx), last_finish = 0.0;
    while (done < n) {
        // admission, in arrival order
        double t = ops->now(ops->ctx);
        while (next < order.size()) {
            const int r = order[next];
            const tmx_request& q = reqs[r];
            if (q.arrival > t) break;
            if (opts->max_active > 0 && (int)active.size() >= opts->max_active) break;
            long long fp = 0;
            int rc = ops->footprint(ops->ctx, &q.c, &fp);
            if (rc == TMX_OK && fp > cap) rc = TMX_E_NOMEM;  // can never fit
            int slot = -1;
            if (rc == TMX_OK) {
                rc = ops->add(ops->ctx, &q.c, &slot);
                if (rc == TMX_E_NOMEM) break;  // wait for a retirement
            }
            if (rc) {  // this request cannot be served; the others go on
                out[r].status = rc;
                out[r].admitted = out[r].finished = t;
                done++;
                next++;
                continue;
            }
            t = ops->now(ops->ctx);
            out[r].slot = slot;
            out[r].admitted = t;
            Active a;
            a.req = r;
            a.slot = slot;
            active.push_back(a);
            next++;
        }
        if (active.empty()) {
            if (next >= order.size()) break;
            const tmx_request& q = reqs[order[next]];
            if (q.arrival > t) {
                ops->wait_until(ops->ctx, q.arrival);
                last_t = ops->now(ops->ctx);
                continue;
            }
            return fail(TMX_E_STATE, "request %d fits the budget but could not be admitted into an empty engine",
                        order[next]);
        }
        most = std::max(most, (int)active.size());
        // one chunk of steps for every admitted mixer
        int rc = ops->step(ops->ctx, every);
        if (rc) return abort_with(rc);
        std::vector<int> slots(active.size());
        for (size_t i = 0; i < active.size(); i++) slots[i] = active[i].slot;
        std::vector<double> im(3 * active.size());
        rc = ops->outlet_im(ops->ctx, slots.data(), (int)slots.size(), im.data());
        if (rc) return abort_with(rc);
        std::vector<int> bad(active.size(), 0);
        if (ops->health) {
            rc = ops->health(ops->ctx, slots.data(), (int)slots.size(), bad.data());
            if (rc) return abort_with(rc);
        }
        checks++;
        const double now = ops->now(ops->ctx);
        area += (now - last_t) * (double)active.size();
        last_t = now;
        std::vector<Active> keep;
        keep.reserve(active.size());
        for (size_t i = 0; i < active.size(); i++) {
            Active& a = active[i];
            const tmx_request& q = reqs[a.req];
            a.steps += every;
            lups += (long long)every * ((long long)q.c.inx * q.c.iny * q.c.nz + (long long)q.c.mnx * q.c.mny * q.c.nz);
            a.history.push_back(std::array<double, 3>{im[3 * i], im[3 * i + 1], im[3 * i + 2]});
            const size_t depth = (size_t)(q.window / every) + 1;
            while (a.history.size() > depth) a.history.pop_front();
            // converged: over the window every index is defined (non-zero:
            // all three species have reached the outlet; the reference
            // reports 0 before) and moved by less than tol
            bool converged = a.history.size() == depth;
            for (size_t h = 0; converged && h < a.history.size(); h++)
                for (int s = 0; s < 3; s++)
                    if (!(a.history[h][s] != 0.0)) converged = false;
            for (int s = 0; converged && s < 3; s++)
                if (!(std::fabs(a.history.back()[s] - a.history.front()[s]) < q.tol)) converged = false;
            if (bad[i] || converged || a.steps >= q.max_steps) {
                tmx_served& o = out[a.req];
                o.status = bad[i] ? TMX_E_NONFINITE : (converged ? 0 : 1);
                o.steps = a.steps;
                o.finished = now;
                for (int s = 0; s < 3; s++) o.outlet_im[s] = a.history.back()[s];
                rc = ops->remove(ops->ctx, a.slot);
                if (rc) {
                    // the failed slot stays the engine's; the others go back
                    for (size_t k = i + 1; k < active.size(); k++) keep.push_back(active[k]);
                    active.swap(keep);
                    return abort_with(rc);
                }
                last_finish = std::max(last_finish, now);
                done++;
            } else {
                keep.push_back(std::move(a));
            }
        }
        active.swap(keep);
    }
    if (summary) {
        std::vector<double> tts;
        for (int r = 0; r < n; r++)
            if (out[r].status == 0 || out[r].status == 1) tts.push_back(out[r].finished - reqs[r].arrival);
        const double makespan = last_finish;
        summary[0] = makespan;
        summary[1] = (double)lups;
        summary[2] = makespan > 0 ? (double)lups / makespan / 1e6 : 0.0;
        summary[3] = nearest_rank(tts, 0.50);
        summary[4] = nearest_rank(tts, 0.99);
        summary[5] = most;
        summary[6] = makespan > 0 ? area / makespan : 0.0;
        summary[7] = (double)checks;
    }
    return TMX_OK;
}

}  // extern "C"

namespace {

struct BatchCtx {
    tmx_batch* b;
    std::chrono::steady_clock::time_point t0;
};

int bf_footprint(void*, const tmx_case* c, long long* bytes) { return tmx_batch_footprint(c, bytes); }
long long bf_capacity(void* ctx)
{
    long long info[8];
    return tmx_batch_info(((BatchCtx*)ctx)->b, info) == TMX_OK ? info[2] : 0;
}
int bf_add(void* ctx, const tmx_case* c, int* slot) { return tmx_batch_add(((BatchCtx*)ctx)->b, c, slot); }
int bf_remove(void* ctx, int slot) { return tmx_batch_remove(((BatchCtx*)ctx)->b, slot); }
int bf_step(void* ctx, int nsteps) { return tmx_batch_step(((BatchCtx*)ctx)->b, nsteps, 1); }
int bf_im(void* ctx, const int* slots, int n, double* im) { return tmx_batch_outlet_im(((BatchCtx*)ctx)->b, slots, n, im); }
int bf_health(void* ctx, const int* slots, int n, int* bad) { return tmx_batch_health(((BatchCtx*)ctx)->b, slots, n, bad); }
double bf_now(void* ctx)
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - ((BatchCtx*)ctx)->t0).count();
}
void bf_wait(void* ctx, double t)
{
    const double d = t - bf_now(ctx);
    if (d > 0) std::this_thread::sleep_for(std::chrono::duration<double>(d));
}

}  // namespace

extern "C" int tmx_serve(tmx_batch* b, const tmx_request* reqs, int n, const tmx_serve_opts* opts, tmx_served* out,
                         double summary[8])
{
    if (!b) return fail(TMX_E_INVALID, "null batch");
    BatchCtx ctx{b, std::chrono::steady_clock::now()};
    tmx_serve_ops ops{&ctx, bf_footprint, bf_capacity, bf_add, bf_remove, bf_step, bf_im, bf_now, bf_wait, bf_health};
    return tmx_serve_with(&ops, reqs, n, opts, out, summary);
}
