// Backend and execution selection (reference: include/backend_selection.hpp).
// The B200 drop-in has no transport: a single rank's neighbor "sends" never
// leave the GPU, and the virtual grid (include/dsx.h) turns them into writes
// into the receiving subdomain's slots.  The names are kept for source
// compatibility.
#pragma once

#include <string_view>

namespace dsdecompx {

enum class BackendKind { Mpi, Nccl, Nvshmem };
enum class BackendSelection { Auto, Mpi, Nccl, Nvshmem };
enum class ExecutionMode { Host, Cuda };

const char* backend_selection_name(BackendSelection selection) noexcept;
BackendSelection parse_backend_selection(std::string_view value);
bool backend_compiled(BackendSelection selection) noexcept;

}  // namespace dsdecompx
