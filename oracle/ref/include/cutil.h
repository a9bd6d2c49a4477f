/* Host-only stand-in for the NVIDIA SDK's cutil timers (the reference only times with them). */
#pragma once
#define cutilCheckError(x) (void)(x)
static inline int cutCreateTimer(unsigned int* t) { *t = 0; return 1; }
static inline int cutResetTimer(unsigned int) { return 1; }
static inline int cutStartTimer(unsigned int) { return 1; }
static inline int cutStopTimer(unsigned int) { return 1; }
static inline float cutGetTimerValue(unsigned int) { return 0.0f; }
