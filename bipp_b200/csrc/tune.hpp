// Tunable launch shapes and work-unit sizes of the kernels: a process-wide table of
// named integer parameters, each with its default and the candidate values the
// autotuner (bipp_autotune_pipeline) times. Launch sites read the current value with
// tuned(); the table can be saved to and loaded from a file (BIPP_B200_TUNING_FILE is
// loaded on first use when set).
#pragma once

#include <vector>

namespace bippb200 {

// current value of the named parameter (throws for an unknown name)
int tuned(const char* name);
// set a parameter to one of its candidates (throws otherwise)
void set_tuned(const char* name, int value);
std::vector<int> tuning_candidates(const char* name);

}  // namespace bippb200
