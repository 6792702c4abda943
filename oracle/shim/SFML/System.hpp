// Oracle test infrastructure only: a self-written stand-in for the two SFML System types the reference
// uses for wall-clock status reports (sf::Clock, sf::Time). SFML is not installed on this image.
#ifndef ORACLE_SHIM_SFML_SYSTEM_HPP
#define ORACLE_SHIM_SFML_SYSTEM_HPP
#include <chrono>

namespace sf {
class Time {
 public:
  explicit Time(double s = 0) : s_(s) {}
  float asSeconds() const { return static_cast<float>(s_); }
  long long asMilliseconds() const { return static_cast<long long>(s_ * 1e3); }

 private:
  double s_;
};
class Clock {
 public:
  Clock() : start_(std::chrono::steady_clock::now()) {}
  Time getElapsedTime() const {
    return Time(std::chrono::duration<double>(std::chrono::steady_clock::now() - start_).count());
  }
  Time restart() {
    Time t = getElapsedTime();
    start_ = std::chrono::steady_clock::now();
    return t;
  }

 private:
  std::chrono::steady_clock::time_point start_;
};
}  // namespace sf
#endif
