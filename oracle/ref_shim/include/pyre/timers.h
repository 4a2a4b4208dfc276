// Minimal stand-in for pyre's timer (test infrastructure): a named wall-clock stopwatch with the
// chained reset().start(), stop() and read() (seconds) that the reference's correlator uses.
#ifndef AMPCOR_REF_SHIM_PYRE_TIMERS_H
#define AMPCOR_REF_SHIM_PYRE_TIMERS_H

#include <chrono>

namespace pyre {

class timer_t {
public:
    explicit timer_t(const char*) {}
    timer_t& reset()
    {
        _elapsed = 0.0;
        return *this;
    }
    timer_t& start()
    {
        _t0 = std::chrono::steady_clock::now();
        return *this;
    }
    timer_t& stop()
    {
        _elapsed += std::chrono::duration<double>(std::chrono::steady_clock::now() - _t0).count();
        return *this;
    }
    double read() const { return _elapsed; }

private:
    std::chrono::steady_clock::time_point _t0{};
    double _elapsed = 0.0;
};

}  // namespace pyre

#endif
