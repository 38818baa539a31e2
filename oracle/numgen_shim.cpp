// Test infrastructure only.  Compiles the reference's NumGen.cpp unmodified
// inside this translation unit so one extra function can rewind its
// per-thread stream counter (an anonymous-namespace variable in
// code/NumGen.cpp:50-53).  A fresh CLI process starts that counter at 0;
// the oracle harness renders many times in one process, so it rewinds it
// before each seeded render to draw the same stream the CLI would.
#include "NumGen.cpp"

extern "C" void pcr_ref_numgen_reset(void)
{
    g_threadCounter.store(0, std::memory_order_relaxed);
}
