// Runs the reference test cases compiled with oracle/kat/capture.h and writes the captured
// known-answer records (one JSON object per line) to argv[1].  Prints the check counts; the
// exit status is the number of failed CHECKs (capped at 255).
#include <cstdio>

#include "capture.h"

int main(int argc, char **argv) {
  std::FILE *out = argc > 1 ? std::fopen(argv[1], "w") : nullptr;
  kat::sink() = out;
  const long failures = doctest::detail::run_all(argc > 2 ? argv[2] : nullptr);
  if (out) std::fclose(out);
  const auto &s = doctest::detail::state();
  std::printf("{\"test_cases\": %zu, \"checks\": %ld, \"failed\": %ld, \"warn_checks\": %ld, "
              "\"warn_failed\": %ld}\n",
              doctest::detail::registry().size(), s.checks, s.failures, s.warn_checks,
              s.warn_failures);
  for (const auto &f : s.failure_log) std::printf("%s\n", f.c_str());
  return failures > 255 ? 255 : static_cast<int>(failures);
}
