// Stand-in for the reference's Parallel (TEST INFRASTRUCTURE): call() runs the target's body for
// every index on the calling thread, the same calls the reference spreads over its threads.
#pragma once
#include <cstddef>
#include "ParallelTarget.hpp"
class Parallel {
public:
    void call(ParallelTarget* target, size_t limit) { for (size_t i = 0; i < limit; i++) target->body(i); }
};
