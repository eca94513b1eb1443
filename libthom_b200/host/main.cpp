// main.cpp — `libthom <test|bench|tune> <routine> ...` (reference: main.cpp:41-72).
#include <stdexcept>
#include <string>
#include <unordered_map>

#include "routines.h"

static const std::unordered_map<std::string, RunMode> runModeMap = {
    {"test", RunMode::TEST}, {"bench", RunMode::BENCH}, {"tune", RunMode::TUNE}};

using RoutineHandler = void (*)(RunMode, int, char**);

// The GEMM routines of this build: `dgemm` and `hgemm` (the reference's routines) and `dgemmb`
// (grouped/batched DGEMM, one persistent launch for many uneven problems).
static const std::unordered_map<std::string, RoutineHandler> routinesMap = {
    {"dgemm", dgemm_handler},
    {"dgemmb", dgemmb_handler},
    {"hgemm", hgemm_handler},
};

int main(int argc, char* argv[]) {
  if (argc < 3) {
    fprintf(stderr, "Not enough parameters, please provide at least ./libthom <test|bench|tune> <ROUTINE>\n");
    return EXIT_FAILURE;
  }
  const char* mode = argv[1];
  const char* routine = argv[2];
  auto m = runModeMap.find(mode);
  auto r = routinesMap.find(routine);
  if (m == runModeMap.end() || r == routinesMap.end()) {
    fprintf(stderr, "Invalid mode or routine: %s %s\nThey must be registered in main.cpp\n", mode, routine);
    return EXIT_FAILURE;
  }
  r->second(m->second, argc, argv);
  return EXIT_SUCCESS;
}
