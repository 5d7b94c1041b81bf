// nvml_energy.cuh -- NVML total-energy counter, loaded at run time with dlopen so the
// library has no link dependency on NVML (NVMLMonitor::read_energy_j,
// src/parallel/nvml_monitor.cpp:85-100 in the reference, replaces its RAPL reading).
// The CUDA device is matched to its NVML handle by PCI bus id.
#pragma once

namespace hamlss {
// Joules consumed by CUDA device `device` since driver load; 0.0 when NVML or the counter
// is missing.
double nvml_energy_j(int device);
// Whether NVML and its energy counter can be read for `device`.
bool nvml_energy_available(int device);
}  // namespace hamlss
