// rmm/resource_ref.hpp -- a device memory resource reference for the groupby
// facade: wraps a gbx_allocator (null: stream-ordered cudaMallocAsync).
#pragma once

#include "../gbx.h"

namespace rmm {

struct device_async_resource_ref {
  gbx_allocator const* allocator{nullptr};
};

namespace mr {
inline device_async_resource_ref get_current_device_resource() { return {}; }
}  // namespace mr

}  // namespace rmm
