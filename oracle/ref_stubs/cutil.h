/* Project-written stand-in for the retired CUDA SDK "cutil" header, used only to
 * compile the reference CPU engine as a test oracle. The reference uses cutil
 * for wall-clock timers (simulation engine/src/Replica.cpp:38-74, :1069-1093;
 * main.cpp:1136-1141) and a checked-call macro. Timers are backed by
 * std::chrono; ids outside the table are ignored, so a timer used before
 * initTimers() is harmless. Test infrastructure only. */
#ifndef REMC_ORACLE_STUB_CUTIL_H
#define REMC_ORACLE_STUB_CUTIL_H

#include <chrono>
#include <cstdio>

/* the SDK macros expand to a statement block, so call sites may omit the
 * trailing semicolon (Replica.cpp:128 does) */
#define CUT_SAFE_CALL(x) { (void)(x); }
#define CUDA_SAFE_CALL(x) { (void)(x); }
#define CUDA_SAFE_CALL_NO_SYNC(x) { (void)(x); }
#define cutilCheckMsg(msg) ((void)0)

namespace remc_stub_timers {
struct Timer {
  bool used;
  bool running;
  double total_ms;
  std::chrono::steady_clock::time_point start;
};
static const unsigned kMax = 4096;
static Timer table[kMax];
static unsigned next_id = 1;
}  // namespace remc_stub_timers

static inline bool cutCreateTimer(unsigned* id) {
  using namespace remc_stub_timers;
  if (next_id >= kMax) { *id = 0; return false; }
  *id = next_id++;
  table[*id].used = true;
  table[*id].running = false;
  table[*id].total_ms = 0.0;
  return true;
}
static inline bool cutDeleteTimer(unsigned id) {
  using namespace remc_stub_timers;
  if (id > 0 && id < kMax) table[id].used = false;
  return true;
}
static inline bool cutStartTimer(unsigned id) {
  using namespace remc_stub_timers;
  if (id == 0 || id >= kMax || !table[id].used) return false;
  table[id].running = true;
  table[id].start = std::chrono::steady_clock::now();
  return true;
}
static inline bool cutStopTimer(unsigned id) {
  using namespace remc_stub_timers;
  if (id == 0 || id >= kMax || !table[id].used || !table[id].running) return false;
  table[id].running = false;
  table[id].total_ms += std::chrono::duration<double, std::milli>(
                            std::chrono::steady_clock::now() - table[id].start).count();
  return true;
}
static inline float cutGetTimerValue(unsigned id) {
  using namespace remc_stub_timers;
  if (id == 0 || id >= kMax || !table[id].used) return 0.0f;
  double t = table[id].total_ms;
  if (table[id].running)
    t += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() -
                                                   table[id].start).count();
  return (float)t;
}
static inline bool cutResetTimer(unsigned id) {
  using namespace remc_stub_timers;
  if (id > 0 && id < kMax) table[id].total_ms = 0.0;
  return true;
}

#endif
