/*
 * Stand-in for gapbs' timer.h (deps/gapbs is an un-vendored submodule of the
 * reference, so src/util.h:13 cannot find it).  Same member names the
 * reference calls: Start, Stop, Seconds, Millisecs.  Built on std::chrono.
 */
#ifndef HC_REF_SHIM_TIMER_H
#define HC_REF_SHIM_TIMER_H
#include <chrono>
class Timer {
public:
    void Start() { t0_ = std::chrono::steady_clock::now(); }
    void Stop() { t1_ = std::chrono::steady_clock::now(); }
    double Seconds() const { return std::chrono::duration<double>(t1_ - t0_).count(); }
    double Millisecs() const { return Seconds() * 1e3; }
    double Microsecs() const { return Seconds() * 1e6; }
private:
    std::chrono::steady_clock::time_point t0_{}, t1_{};
};
#endif
