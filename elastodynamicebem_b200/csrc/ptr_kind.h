// Classification of a caller's buffer for the C ABI, free of CUDA headers so
// that it compiles (and is unit-tested) on a machine without a GPU.
//
// mem_type takes the values of cudaMemoryType (0 unregistered host memory,
// 1 registered / pinned host memory, 2 device memory, 3 managed memory);
// ptr_device is the device that owns device memory and current_device the
// device the call runs on (the mesh's device for mesh-based entry points).
#pragma once

namespace ebem {

enum class PtrKind {
    Host,         // staged through device memory by the library
    Device,       // used in place by the call's kernels
    OtherDevice,  // device memory of another GPU: rejected (a kernel on the
                  // call's device would fault on it without peer access)
};

inline PtrKind classify_pointer(int mem_type, int ptr_device, int current_device) {
    if (mem_type == 2) return ptr_device == current_device ? PtrKind::Device : PtrKind::OtherDevice;
    if (mem_type == 3) return PtrKind::Device;     // managed memory is reachable from every device
    return PtrKind::Host;
}

}  // namespace ebem
