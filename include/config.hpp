// Decomp configuration (reference: include/config.hpp).
#pragma once

#include "backend_selection.hpp"
#include "domain.hpp"
#include "grid.hpp"

#include <cstddef>

namespace dsdecompx {

// AdvancedBackendConfig::cuda_device besides an explicit ordinal
constexpr int kCudaDeviceCurrent = -1;
constexpr int kCudaDeviceByLocalRank = -2;

struct AdvancedBackendConfig {
    BackendSelection selection = BackendSelection::Auto;
    bool read_environment = true;
    bool allow_host_staging = true;
    int cuda_device = kCudaDeviceCurrent;
};

struct DynamicLoadBalanceConfig {
    std::size_t interval = 1;            // rebalance every N migrate() calls; 0 disables
    double imbalance_threshold = 1.10;   // max(work) / mean(work) that triggers it
    double relaxation = 0.5;             // fraction of the proposed cut move applied
    double minimum_cell_fraction = 0.10; // smallest cell as a fraction of a uniform one
};

struct Config {
    GlobalDomain domain;
    ProcessGrid process_grid;
    HaloConfig halo;
    GridPolicy grid_policy = GridPolicy::Manual;
    TopologyInfo topology_info;
    DynamicLoadBalanceConfig dynamic;
    ExecutionMode execution = ExecutionMode::Cuda;
    AdvancedBackendConfig advanced;
};

struct MigrationResult {
    bool ownership_changed = false;
    std::size_t previous_owned_count = 0;
    std::size_t retained_count = 0;
    std::size_t sent_count = 0;
    std::size_t received_count = 0;
    std::size_t new_owned_count = 0;
};

}  // namespace dsdecompx
