// Host helpers of mcstar-libs common/technicalities.hpp:3-32: stream output and
// equality of the CUDA vector types, and shape_tr, the numpy-order (slowest first)
// shape of an x-fastest extent.
#pragma once
#include <cuda_runtime.h>

#include <ostream>
#include <stdexcept>

inline std::ostream& operator<<(std::ostream& o, const dim3& v) { return o << v.x << ' ' << v.y << ' ' << v.z; }
inline std::ostream& operator<<(std::ostream& o, const float3& v) { return o << v.x << ' ' << v.y << ' ' << v.z; }
inline std::ostream& operator<<(std::ostream& o, const double3& v) { return o << v.x << ' ' << v.y << ' ' << v.z; }
inline std::ostream& operator<<(std::ostream& o, const int3& v) { return o << v.x << ' ' << v.y << ' ' << v.z; }
inline std::ostream& operator<<(std::ostream& o, const float2& v) { return o << v.x << ' ' << v.y; }
inline std::ostream& operator<<(std::ostream& o, const double2& v) { return o << v.x << ' ' << v.y; }
inline std::ostream& operator<<(std::ostream& o, const int2& v) { return o << v.x << ' ' << v.y; }

inline bool operator==(const int3& a, const int3& b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
inline bool operator==(const uint3& a, const uint3& b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
inline bool operator==(const int2& a, const int2& b) { return a.x == b.x && a.y == b.y; }
inline bool operator==(const uint2& a, const uint2& b) { return a.x == b.x && a.y == b.y; }

// x-fastest extent -> numpy shape: (nx) for 1D, (ny, nx) for 2D, (nz, ny, nx) for 3D
inline int3 shape_tr(int3 in) {
    if (in.z != 1) return int3{in.z, in.y, in.x};
    if (in.y != 1) return int3{in.y, in.x, 1};
    return int3{in.x, 1, 1};
}
