// Host worker pool for the host-side copies of the API (staging IR rows from
// the caller's pageable buffers into pinned memory). One pool per process,
// started on first use; the calling thread takes part in every job.
#pragma once

#include <cstddef>
#include <functional>

namespace tanb {

// Runs fn(i) for i in [0, n), spread over the pool's threads and the caller;
// returns when all calls have finished. Calls of fn must be independent.
void host_parallel_for(int n, const std::function<void(int)>& fn);

// Worker threads of the pool (0 until first use), for reporting.
int host_pool_threads();

}  // namespace tanb
