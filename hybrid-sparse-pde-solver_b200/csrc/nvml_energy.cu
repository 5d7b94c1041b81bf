// nvml_energy.cu -- see nvml_energy.cuh.  Reads only; never changes a GPU setting.
#include <dlfcn.h>

#include <cuda_runtime.h>

#include <mutex>

#include "nvml_energy.cuh"

namespace hamlss {

namespace {
typedef int (*fn_init)(void);
typedef int (*fn_by_bus)(const char*, void**);
typedef int (*fn_energy)(void*, unsigned long long*);

constexpr int kMaxDevices = 64;

struct Nvml {
    bool ok = false;
    fn_by_bus by_bus = nullptr;
    fn_energy energy = nullptr;
    std::mutex mu;
    void* handle[kMaxDevices] = {};
    bool looked_up[kMaxDevices] = {};
    Nvml() {
        void* lib = dlopen("libnvidia-ml.so.1", RTLD_LAZY | RTLD_LOCAL);
        if (!lib) return;
        auto init = (fn_init)dlsym(lib, "nvmlInit_v2");
        by_bus = (fn_by_bus)dlsym(lib, "nvmlDeviceGetHandleByPciBusId_v2");
        energy = (fn_energy)dlsym(lib, "nvmlDeviceGetTotalEnergyConsumption");
        ok = init && by_bus && energy && init() == 0;
    }
    // NVML numbers devices in PCI order over all GPUs of the machine; a CUDA ordinal
    // follows CUDA_VISIBLE_DEVICES and CUDA_DEVICE_ORDER.  The PCI bus id names the same
    // GPU in both, so the handle is looked up by it (once per CUDA device).
    void* device_handle(int device) {
        if (device < 0 || device >= kMaxDevices) return nullptr;
        std::lock_guard<std::mutex> g(mu);
        if (!looked_up[device]) {
            looked_up[device] = true;
            char bus[32] = {};
            if (cudaDeviceGetPCIBusId(bus, (int)sizeof(bus), device) == cudaSuccess) {
                void* h = nullptr;
                if (by_bus(bus, &h) == 0) handle[device] = h;
            } else {
                cudaGetLastError();      // clear the failed query so no later launch check reports it
            }
        }
        return handle[device];
    }
};

Nvml& nvml() {
    static Nvml n;
    return n;
}
}  // namespace

bool nvml_energy_available(int device) {
    Nvml& n = nvml();
    return n.ok && n.device_handle(device) != nullptr;
}

double nvml_energy_j(int device) {
    Nvml& n = nvml();
    if (!n.ok) return 0.0;
    void* h = n.device_handle(device);
    if (!h) return 0.0;
    unsigned long long mj = 0;
    if (n.energy(h, &mj) != 0) return 0.0;
    return (double)mj * 1e-3;
}

}  // namespace hamlss
