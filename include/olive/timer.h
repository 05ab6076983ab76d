/*
 * olive_b200 source-compatible header layer: wall-clock helpers with the
 * reference's names (timer.h:41-74).  Uses a monotonic clock.
 */
#ifndef OLIVE_TIMER_H
#define OLIVE_TIMER_H

#include <time.h>

inline double getTimeMillis() {
    timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return t.tv_sec * 1000.0 + t.tv_nsec / 1e6;
}

inline double getTimeSeconds() { return getTimeMillis() / 1000.0; }

/** Lap timer: getElapsedMillis() returns the time since the previous call. */
class Stopwatch {
    double last_ = 0;

public:
    void start() { last_ = getTimeMillis(); }
    double getElapsedMillis() {
        double now = getTimeMillis();
        double d = now - last_;
        last_ = now;
        return d;
    }
};

#endif  // OLIVE_TIMER_H
