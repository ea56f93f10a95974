// loadgen.cpp — libnbgpu_loadgen.so: an open-loop request generator for the
// serving benchmark.  It submits device-resident requests to an nbg_server at
// given arrival times (seconds after a start instant), spinning on the clock
// between arrivals, so the offered rate is limited by nbg_submit_dev itself
// (about a microsecond) rather than by an interpreter loop.  Not part of the
// product: the benchmark loads it beside libnbgpu.so.
#include <chrono>
#include <cstdint>

#include "../../include/nbgpu.h"

extern "C" {

// Submits requests i = 0..count-1: request i is pool[order[i]] and is
// submitted when t_start_s + arrival_s[i] is reached on the steady clock
// (t_start_s from nbg_loadgen_now).  tickets[i] gets its ticket and lag_us[i]
// how late it was submitted.  Returns NBG_OK, or the first nbg_submit_dev
// error (the requests before it were submitted; *done tells how many).
int nbg_loadgen_submit(nbg_server* s, const nbg_desc* pool, const int32_t* order, const double* arrival_s,
                       int64_t count, double t_start_s, int64_t* tickets, double* lag_us, int64_t* done) {
    using clk = std::chrono::steady_clock;
    *done = 0;
    for (int64_t i = 0; i < count; i++) {
        const double due = t_start_s + arrival_s[i];
        double now = std::chrono::duration<double>(clk::now().time_since_epoch()).count();
        while (now < due) now = std::chrono::duration<double>(clk::now().time_since_epoch()).count();
        int rc = nbg_submit_dev(s, &pool[order[i]], &tickets[i]);
        if (rc != NBG_OK) return rc;
        lag_us[i] = (now - due) * 1e6;
        *done = i + 1;
    }
    return NBG_OK;
}

// The steady clock in seconds (the time base of nbg_loadgen_submit).
double nbg_loadgen_now(void) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // extern "C"
