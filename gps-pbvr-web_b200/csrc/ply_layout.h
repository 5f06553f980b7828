// Layout of a 3DGS PLY's vertex records (shared by the host loader and the GPU decoder).
#pragma once
#include <stddef.h>
#include <stdint.h>

#include "../../include/gpsb200.h"

namespace gpsb {

// Property order: x y z f_dc_0..2 opacity scale_0..2 rot_0..3 (14) then f_rest_0.. (0, 9, 24, 45).
// type: 0 int8, 1 uint8, 2 int16, 3 uint16, 4 int32, 5 uint32, 6 float32, 7 float64 (little endian).
struct PlyLayout {
    bool binary = false;
    size_t count = 0, stride = 0, data_start = 0;
    uint32_t degree = 0, nprop = 0;
    uint32_t off[59];
    uint8_t type[59];
};

gpsb_status ply_layout(const uint8_t* bytes, size_t len, PlyLayout* out);
gpsb_status ply_error(const char* msg);  // sets gpsb_ply_last_error, returns GPSB_ERR_PARSE

}  // namespace gpsb
