#pragma once

namespace dsdecompx {
inline constexpr int version_major = 1;
inline constexpr int version_minor = 0;
inline constexpr int version_patch = 0;
inline constexpr const char* version_string = "1.0.0";
}  // namespace dsdecompx
