// device_slots.h -- per-device slots of a per-thread cache (host code).
//
// The reference-compatible entry points keep device buffers between calls
// (a workspace, a device copy of the caller's LUT).  They run on the calling
// thread's current device, so a cached buffer is only ever handed to calls
// on the device it was allocated on: the cache holds one slot per device
// index and each slot remembers its device (the slot's destructor frees the
// buffers there).
#pragma once

namespace tops {

template <class T, int N>
struct DeviceSlots {
  T slot[N];
  // The slot of device `dev`, tagged with it; null for an index outside
  // 0 .. N - 1.
  T *at(int dev) {
    if (dev < 0 || dev >= N) return nullptr;
    slot[dev].dev = dev;
    return &slot[dev];
  }
};

}  // namespace tops
