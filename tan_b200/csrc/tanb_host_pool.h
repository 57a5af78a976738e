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

// memcpy into pinned memory that the device reads next (a host-to-device copy
// or a kernel reading mapped host memory). On x86-64, copies of 4 KiB and more
// use non-temporal stores, followed by a store fence: lines written through
// the cache stay dirty there, and a device read of dirty lines is served from
// the CPU's caches at a fraction of the bus rate (a 16 MiB upload measured
// 2.2x slower end to end); non-temporal stores leave nothing in the cache.
void copy_for_device(void* dst, const void* src, size_t bytes);

// The same for many short rows: non-temporal stores from 256 bytes on and no
// fence; the thread calls copy_for_device_fence() once after its last row.
void copy_rows_for_device(void* dst, const void* src, size_t bytes);
void copy_for_device_fence();

}  // namespace tanb
