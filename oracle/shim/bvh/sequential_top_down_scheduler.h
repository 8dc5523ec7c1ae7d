// Test infrastructure (oracle): scheduler tag types (the build itself decides
// how to parallelise).
#pragma once
namespace bvh { template <typename Builder> struct SequentialTopDownScheduler {}; }
