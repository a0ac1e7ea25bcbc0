// Exercises sp::HostPool (the scan's host thread pool) without a GPU: every index of every
// round runs exactly once, rounds follow one another with and without pauses long enough
// for the workers to fall asleep, and a task's exception reaches the caller after the
// round has finished.
#include <cstdio>
#include <stdexcept>
#include <vector>

#include "host_pool.hpp"

int main() {
  sp::HostPool pool(7);
  std::vector<int> hits(1000, 0);
  for (int round = 0; round < 2000; ++round) {
    pool.run(1000, [&](int i) { hits[i] += 1; });
    if (round % 100 == 0) std::this_thread::sleep_for(std::chrono::milliseconds(1));
  }
  for (int h : hits)
    if (h != 2000) {
      std::printf("an index ran %d times in 2000 rounds\n", h);
      return 1;
    }
  std::vector<int> ran(100, 0);
  bool caught = false;
  try {
    pool.run(100, [&](int i) {
      ran[i] = 1;
      if (i == 37) throw std::runtime_error("task 37");
    });
  } catch (const std::runtime_error&) {
    caught = true;
  }
  if (!caught) {
    std::printf("the task's exception did not reach the caller\n");
    return 1;
  }
  for (int r : ran)
    if (!r) {
      std::printf("a task was skipped after another one threw\n");
      return 1;
    }
  sp::HostPool alone(0);
  int sum = 0;
  alone.run(10, [&](int i) { sum += i; });
  if (sum != 45) return 1;
  std::printf("ok\n");
  return 0;
}
