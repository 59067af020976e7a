// Host build of the library's procedural sky (rt_sky.cuh), for the CPU
// parity test against the reference's own sky sampler.  Test-only.
#include <cstddef>
#include <cstring>

#include "rt_sky.cuh"

extern "C" void host_sample_sky(const void* profile, double x, double y, double z, double fov, double time,
                                float out[3]) {
    relsim::SkyProfile p;
    std::memcpy(&p, profile, sizeof p);
    relsim::sky::sample(p, x, y, z, fov, time, out);
}

// Byte offset of a field (kind 0: uint32, 1: double, 2: float[4] vector or the
// grid cell colour table); -1 if unknown.
extern "C" long host_sky_offset(const char* name, int* kind) {
#define RT_SKY_FIND(T, N, D)                                    \
    if (std::strcmp(name, #N) == 0) {                           \
        *kind = (sizeof(T) == 8) ? 1 : 0;                       \
        return static_cast<long>(offsetof(relsim::SkyProfile, N)); \
    }
    RT_SKY_U32_FIELDS(RT_SKY_FIND)
    RT_SKY_F64_FIELDS(RT_SKY_FIND)
#undef RT_SKY_FIND
#define RT_SKY_FIND_VEC(N, A, B, C)                             \
    if (std::strcmp(name, #N) == 0) {                           \
        *kind = 2;                                              \
        return static_cast<long>(offsetof(relsim::SkyProfile, N)); \
    }
    RT_SKY_VEC_FIELDS(RT_SKY_FIND_VEC)
#undef RT_SKY_FIND_VEC
    if (std::strcmp(name, "grid_cell_colors") == 0) {
        *kind = 2;
        return static_cast<long>(offsetof(relsim::SkyProfile, grid_cell_colors));
    }
    return -1;
}
