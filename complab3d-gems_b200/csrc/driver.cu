// driver.cu -- the coupled step driven as the reference's main loop drives it (complab.cpp:2178-3262).
//
// One call advances `iterations` transport iterations of a domain whose lattices, kinetics,
// automaton and precipitation were set up through the other entry points. Per iteration, in the
// reference's order:
//   1. collide every mobile species, biotic then abiotic kinetics with the clamp, speciation,
//      stream (complab.cpp:2307-2569, 3251-3259): one fused clb_ade_step;
//   2. the biofilm automaton (complab.cpp:2792-3055): clb_ca_step;
//   3. when it changed the mask (complab.cpp:3073-3135): the species dynamics follow it at
//      iterations that are multiples of ade_update_interval, the flow dynamics follow it and the
//      flow is re-solved and coupled again at multiples of ns_update_interval;
//   4. precipitation / dissolution node conversion at multiples of the precipitation interval,
//      with its own flow re-solve when voxels sealed or reopened (complab.cpp:3139-3247):
//      clb_geometry_update.
// Besides the reference's schedule, `resolve_every` re-solves the flow unconditionally every that
// many iterations (after the mask changed since the previous re-solve, the flow dynamics follow it
// first), which is how a parameter study states "flow re-solved every 500 steps".
//
// The run stops where the reference stops (percolationFlag, complab.cpp:2796, 3113, 3117):
// non-finite values (CLB_NONFINITE), a sealed flow path (CLB_PERCOLATION_LOST), a biofilm push
// that cannot settle (CLB_NOT_CONVERGED from the automaton). A flow re-solve that reaches its cap
// while the outlet still flows is counted and the run continues, as the reference continues
// after its warning (complab.cpp:3100-3112).
//
// The report carries counts and the device time of each phase, measured with CUDA events on the
// handle's stream around the phase's launches (the transport time is the fused step's own).
#include "clb_internal.cuh"

#include <chrono>
#include <cstring>
#include <vector>

namespace clb {

namespace {

// Device time accumulated over the phases of a run: an event pair per phase occurrence, recorded
// on the handle's stream without waiting; the pairs are summed once the run has synchronised.
struct PhaseTimer {
    cudaStream_t s;
    std::vector<cudaEvent_t> ev;  // pairs (start, stop)
    size_t used = 0;
    bool ok = true;
    explicit PhaseTimer(cudaStream_t st) : s(st) {}
    ~PhaseTimer() {
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
    }
    cudaEvent_t next() {
        if (used == ev.size()) {
            cudaEvent_t e = nullptr;
            if (cudaEventCreate(&e) != cudaSuccess) { ok = false; return nullptr; }
            ev.push_back(e);
        }
        return ev[used++];
    }
    void start() {
        if (used & 1) return;  // unmatched start: keep the first
        cudaEvent_t e = next();
        if (e) cudaEventRecord(e, s);
    }
    void stop() {
        if (!(used & 1)) return;
        cudaEvent_t e = next();
        if (e) cudaEventRecord(e, s);
    }
    // total of the recorded pairs in ms (synchronises on the last event)
    double total() {
        if (!ok || used < 2) return 0.0;
        cudaEventSynchronize(ev[used - 1]);
        double acc = 0.0;
        for (size_t i = 0; i + 1 < used; i += 2) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, ev[i], ev[i + 1]) == cudaSuccess) acc += ms;
        }
        return acc;
    }
};

}  // namespace

static clb_status resolve_flow(clb_handle* h, const clb_run_desc* d, bool mask_moved, clb_run_report* r,
                               PhaseTimer& t) {
    t.start();
    clb_status st = CLB_OK;
    if (mask_moved && h->ca_ready) st = refresh_dynamics(h, 0, 1);  // updateNsLatticesDynamics3D
    int it = 0;
    if (st == CLB_OK) st = flow_solve(h, d->flow_max_iterations, d->flow_eps, &it, true);
    r->flow_resolves += 1;
    r->flow_iterations += it;
    if (st == CLB_NOT_CONVERGED) {
        r->flow_unconverged += 1;  // the outlet still flows: warn and go on, as the reference does
        st = CLB_OK;
    }
    if (st == CLB_OK) st = ade_couple(h);  // latticeToPassiveAdvDiff
    t.stop();
    return st;
}

clb_status run(clb_handle* h, const clb_run_desc* d, clb_run_report* r) {
    std::memset(r, 0, sizeof(*r));
    if (!h->ade_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ade_init first");
    if (d->iterations < 0 || d->ade_update_interval < 0 || d->ns_update_interval < 0 || d->resolve_every < 0 ||
        d->geometry_interval < 0 || d->flow_max_iterations < 0)
        return fail(h, CLB_INVALID_ARG, "negative count or interval");
    if (d->ca && !h->ca_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_ca_setup first (ca = 1)");
    if (d->geometry_interval && !h->prc_ready) return fail(h, CLB_NOT_INITIALIZED, "clb_precip_setup first");
    const bool resolves = (d->ns_update_interval > 0 || d->resolve_every > 0);
    if (resolves && !h->flow_ready) return fail(h, CLB_NOT_INITIALIZED, "flow re-solves need clb_flow_init");
    if (resolves && !(d->flow_eps > 0) && d->flow_max_iterations <= 0)
        return fail(h, CLB_INVALID_ARG, "a flow re-solve needs flow_eps > 0 or an iteration cap");
    const auto wall0 = std::chrono::steady_clock::now();
    const int64_t launches0 = h->launches;
    PhaseTimer tt(h->stream), tc(h->stream), tf(h->stream), tg(h->stream);
    bool moved_since_resolve = false;
    clb_status st = CLB_OK;
    // The automaton's steps run on the device without the host in the loop unless a schedule needs
    // each step's outcome on the host at once (a re-solve on a mask change, abiotic laws whose lists
    // follow the map): the dynamics refresh after a mask change is enqueued every update interval
    // and acts only when the step changed the mask, and the results (failures, counts) are read
    // back every POLL iterations, at each re-solve and at the end.
    const bool ca_async = d->ca && d->ns_update_interval == 0 && h->ap.law2 == CLB_LAW_NONE && !h->ap.dis_on;
    constexpr int POLL = 64;
    int64_t ca_sweeps0 = 0, ca_changes0 = 0, ca_changes_at_resolve = 0;
    if (ca_async) {
        st = ca_read(h, nullptr, nullptr, &ca_sweeps0, &ca_changes0);
        ca_changes_at_resolve = ca_changes0;
    }
    auto ca_poll = [&](bool for_resolve) {
        int64_t sw = 0, ch = 0;
        clb_status ps = ca_read(h, nullptr, nullptr, &sw, &ch);
        r->ca_sweeps = (int)(sw - ca_sweeps0);
        r->mask_changes = (int)(ch - ca_changes0);
        if (for_resolve) {
            if (ch != ca_changes_at_resolve) moved_since_resolve = true;
            ca_changes_at_resolve = ch;
        }
        if (ps == CLB_OK) ps = ade_nonfinite_check(h);
        return ps;
    };
    for (int k = 0; k < d->iterations && st == CLB_OK; ++k) {
        const int64_t iT = h->ade_iters;  // the reference's iteration counter at this step
        tt.start();
        st = ade_step(h, 1);
        tt.stop();
        if (st != CLB_OK) break;
        r->iterations += 1;
        if (ca_async) {
            tc.start();
            st = ca_step_async(h, iT);
            if (st == CLB_OK && d->ade_update_interval > 0 && iT % d->ade_update_interval == 0)
                st = refresh_species_if_changed(h);  // updateSoluteDynamics3D after a mask change
            tc.stop();
            if (st != CLB_OK) break;
            if ((k + 1) % POLL == 0 && (st = ca_poll(false)) != CLB_OK) break;
        } else if (d->ca) {
            int sweeps = 0, changed = 0;
            tc.start();
            st = ca_step(h, &sweeps, &changed);  // synchronises: its mask pass reads counters back
            tc.stop();
            r->ca_sweeps += sweeps;
            if (st != CLB_OK) break;
            if ((st = ade_nonfinite_check(h)) != CLB_OK) break;  // the step before has completed
            if (changed) {
                r->mask_changes += 1;
                moved_since_resolve = true;
                if (d->ade_update_interval > 0 && iT % d->ade_update_interval == 0) {
                    tc.start();
                    st = refresh_dynamics(h, 1, 0);  // updateSoluteDynamics3D
                    tc.stop();
                    if (st != CLB_OK) break;
                }
                if (d->ns_update_interval > 0 && iT % d->ns_update_interval == 0) {
                    st = resolve_flow(h, d, true, r, tf);
                    moved_since_resolve = false;
                    if (st != CLB_OK) break;
                }
            }
        }
        if (d->resolve_every > 0 && (iT + 1) % d->resolve_every == 0) {
            if (ca_async && (st = ca_poll(true)) != CLB_OK) break;
            if ((st = ade_nonfinite_check(h)) != CLB_OK) break;
            st = resolve_flow(h, d, moved_since_resolve, r, tf);
            moved_since_resolve = false;
            if (st != CLB_OK) break;
        }
        if (d->geometry_interval > 0 && iT % d->geometry_interval == 0) {
            int sealed = 0, reopened = 0;
            tg.start();
            st = geometry_update(h, &sealed, &reopened);
            tg.stop();
            r->sealed += sealed;
            r->reopened += reopened;
            if (st == CLB_NOT_CONVERGED) {
                r->flow_unconverged += 1;
                st = CLB_OK;
            }
            if (st != CLB_OK) break;
        }
    }
    tt.stop();
    tc.stop();
    tg.stop();
    tf.stop();
    if (ca_async) {
        const clb_status ps = ca_poll(false);
        if (st == CLB_OK) st = ps;
    }
    const cudaError_t e = cudaStreamSynchronize(h->stream);
    r->ms_transport = tt.total();
    r->ms_ca = tc.total();
    r->ms_flow = tf.total();
    r->ms_geometry = tg.total();
    r->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - wall0).count();
    r->launches = h->launches - launches0;
    if (st != CLB_OK) return st;
    if (e != cudaSuccess) return cuda_check(h, e, "run");
    return ade_nonfinite_check(h);
}

}  // namespace clb
