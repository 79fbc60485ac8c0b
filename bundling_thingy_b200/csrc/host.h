// host.h — host-side pieces of the library (loader, geometry readers).
#pragma once

#include <stddef.h>
#include <stdint.h>

#include <string>
#include <vector>

namespace bt {

struct HostGraph {
    std::vector<float> xy;          // 2 floats per control point
    std::vector<uint32_t> starts;   // edges + 1
    float min[2], max[2];
};

bool parse_trl(const char* text, size_t len, HostGraph* g, std::string* err);
bool load_trl(const char* path, HostGraph* g, std::string* err);
bool normalization(const float mn[2], const float mx[2], float out[5], std::string* err);

// src/geometry.rs:28-73, 107-118
bool layout_check(const uint32_t* paths, uint32_t n_paths, uint32_t samples, std::string* err);
// src/geometry.rs:131-187
bool decode_points(const uint32_t* paths, uint32_t n_paths, uint32_t samples, const void* records, size_t bytes,
                   float* xy, std::string* err);
// src/distortion.rs:137-168
bool squared_integral_host(const float* original, size_t n_original, const float* current, size_t n_current,
                           double* out, std::string* err);

// Kahan-compensated sum (src/distortion.rs:118-131).
struct KahanSum {
    double value = 0.0, correction = 0.0;
    void add(double term) {
        const double adjusted = term - correction;
        const double next = value + adjusted;
        correction = (next - value) - adjusted;
        value = next;
    }
};

}  // namespace bt
