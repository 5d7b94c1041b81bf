// nvml_energy.cu -- see nvml_energy.cuh.  Reads only; never changes a GPU setting.
#include <dlfcn.h>

#include <mutex>

#include "nvml_energy.cuh"

namespace hamlss {

namespace {
typedef int (*fn_init)(void);
typedef int (*fn_handle)(unsigned, void**);
typedef int (*fn_energy)(void*, unsigned long long*);

struct Nvml {
    bool ok = false;
    fn_handle handle = nullptr;
    fn_energy energy = nullptr;
    Nvml() {
        void* lib = dlopen("libnvidia-ml.so.1", RTLD_LAZY | RTLD_LOCAL);
        if (!lib) return;
        auto init = (fn_init)dlsym(lib, "nvmlInit_v2");
        handle = (fn_handle)dlsym(lib, "nvmlDeviceGetHandleByIndex_v2");
        energy = (fn_energy)dlsym(lib, "nvmlDeviceGetTotalEnergyConsumption");
        ok = init && handle && energy && init() == 0;
    }
};

Nvml& nvml() {
    static Nvml n;
    return n;
}
}  // namespace

double nvml_energy_j(int device) {
    Nvml& n = nvml();
    if (!n.ok) return 0.0;
    void* h = nullptr;
    if (n.handle((unsigned)device, &h) != 0) return 0.0;
    unsigned long long mj = 0;
    if (n.energy(h, &mj) != 0) return 0.0;
    return (double)mj * 1e-3;
}

}  // namespace hamlss
