// Tracing hooks.  The reference marks its hot functions with
// vampir_trace<N> objects (boost/numeric/mtl/interface/vpt.hpp:37-78): a
// numeric event id per function (names in interface/vpt.cpp, e.g. 7004
// "bicgstab", 5038 "ilu_0::factorize", 3049 "crs_cvec_mult") whose scope is
// an entry/exit pair for the tracer.  Here a TraceScope at the same places
// (same ids where the reference has one; 9xxx for steps the reference does
// not have: preconditioner set-up phases, refinement, batches, serving)
//   * pushes an NVTX range "<id> <name>" for the scope (Nsight Systems,
//     ncu --nvtx filters), and
//   * while tracing is on (mtlg_trace_enable, or MTLG_TRACE=1 in the
//     environment at first use) adds the scope's host wall time to a tally
//     per event, read back with mtlg_trace_report.
// Scopes that end in a stream synchronization (preconditioner set-up,
// solves that report a result) include the device time; others measure
// only the enqueue.
#pragma once
#include <nvtx3/nvToolsExt.h>

#include <chrono>
#include <cstdlib>
#include <map>
#include <mutex>
#include <optional>
#include <string>

namespace mtlg {

struct TraceTally {
    std::string name;
    long long calls = 0;
    double seconds = 0.0;
};

struct TraceState {
    std::mutex mu;
    std::map<int, TraceTally> events;
    int on = -1;   // -1: not yet read from the environment
};

inline TraceState& trace_state()
{
    static TraceState s;
    return s;
}

inline bool trace_on()
{
    TraceState& s = trace_state();
    if (s.on < 0) {
        const char* e = std::getenv("MTLG_TRACE");
        s.on = (e && *e && *e != '0') ? 1 : 0;
    }
    return s.on == 1;
}

class TraceScope {
  public:
    TraceScope(int id, const char* name) : id_(id), name_(name), timed_(trace_on())
    {
        char buf[96];
        snprintf(buf, sizeof buf, "%d %s", id, name);
        nvtxRangePushA(buf);
        if (timed_) t0_ = std::chrono::steady_clock::now();
    }
    ~TraceScope()
    {
        nvtxRangePop();
        if (!timed_) return;
        const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
        TraceState& s = trace_state();
        std::lock_guard<std::mutex> lk(s.mu);
        TraceTally& t = s.events[id_];
        t.name = name_;
        t.calls += 1;
        t.seconds += dt;
    }
    TraceScope(const TraceScope&) = delete;
    TraceScope& operator=(const TraceScope&) = delete;

  private:
    int id_;
    const char* name_;
    bool timed_;
    std::chrono::steady_clock::time_point t0_;
};

// Consecutive phases of one function: next() closes the running phase's
// scope and opens the next one.
class TracePhases {
  public:
    void next(int id, const char* name)
    {
        cur_.reset();
        cur_.emplace(id, name);
    }
    void end() { cur_.reset(); }

  private:
    std::optional<TraceScope> cur_;
};

#define MTLG_TRACE_CAT2(a, b) a##b
#define MTLG_TRACE_CAT(a, b) MTLG_TRACE_CAT2(a, b)
#define MTLG_TRACE(id, name) ::mtlg::TraceScope MTLG_TRACE_CAT(mtlg_trace_scope_, __LINE__)(id, name)

}  // namespace mtlg
