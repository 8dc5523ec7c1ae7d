// Test infrastructure (oracle): scheduler tag type.
#pragma once
namespace bvh::omp { template <typename Builder> struct ParallelTopDownScheduler {}; }
