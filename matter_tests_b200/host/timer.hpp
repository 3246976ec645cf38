// timer.hpp — wall-clock stopwatch with the interface of the reference's
// src/timer.hpp (start, stop, get_timing in seconds).
#ifndef TIMER_HPP
#define TIMER_HPP
#include <chrono>

class timer {
 public:
  void start() { t0_ = std::chrono::steady_clock::now(); }
  void stop() { t1_ = std::chrono::steady_clock::now(); }
  double get_timing() const { return std::chrono::duration<double>(t1_ - t0_).count(); }

 private:
  std::chrono::steady_clock::time_point t0_{}, t1_{};
};

#endif
