// Depth-sorted alpha path (crates/gps-render/src/sorted.rs; shaders/gps_sort.wgsl,
// gps_sorted_draw.wgsl, sp_project / sp_resolve of gps_splat.wgsl) and the onesweep radix sort.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "internal.h"

typedef unsigned long long ull_t;

namespace gpsb {

// Device scratch of one radix sort of n (key, value) pairs.
struct RadixScratch {
    void* hist = nullptr;      // passes x bins u32 global digit histograms (exclusive after the scan)
    void* lookback = nullptr;  // passes x tiles x bins u32 chained-scan words
    void* counters = nullptr;  // passes u32 tile counters
    size_t hist_bytes = 0, lookback_bytes = 0;
    uint32_t cap_n = 0, cap_bins = 0, cap_passes = 0;
};
void radix_release(RadixScratch& s);
// Stable ascending LSD sort of `n` pairs on the low `key_bits` bits with `digit_bits` (4, 6 or 8)
// per pass. Sorted pairs end in (keys_out, vals_out); keys_in/vals_in are used as ping-pong
// buffers and are clobbered.
cudaError_t radix_sort_pairs(RadixScratch& s, uint32_t* keys_in, uint32_t* vals_in, uint32_t* keys_out,
                             uint32_t* vals_out, uint32_t n, int key_bits, int digit_bits, uint32_t* err,
                             cudaStream_t st);

struct SortedState {
    uint32_t cap_n = 0, cap_entries = 0, W = 0, H = 0, tw = 16, th = 16;
    void* keys_a = nullptr;   // n u32
    void* vals_a = nullptr;
    void* keys_b = nullptr;   // sorted keys (the test hook)
    void* vals_b = nullptr;   // sorted splat ids
    void* rec = nullptr;      // n x 3 float4: (mean, o, K), (w1, w2), (rgb, -)
    void* tiles = nullptr;    // n x uint2: tile rectangle of the splat (packed), 0 when invalid
    void* cnt = nullptr;      // n u32 tiles touched, in sorted order, then exclusive offsets
    void* scan_scratch = nullptr;
    size_t scan_scratch_bytes = 0;
    void* ent_key_a = nullptr; void* ent_val_a = nullptr;   // tile entries (tile id, sorted rank)
    void* ent_key_b = nullptr; void* ent_val_b = nullptr;
    void* ranges = nullptr;   // n_tiles x uint2 [start, end)
    void* host_total = nullptr;  // pinned u32
    uint32_t n_tiles = 0;
    int digit_bits = 8;
    RadixScratch rs_keys, rs_tiles;
};
void sorted_release(SortedState& s);
// Projects, sorts and blends (full = true, writes accum = (rgb, 1)) or only probes the GPS
// particle demand into stats[ST_PROBE] (full = false).
cudaError_t sorted_render(SortedState& s, const FrameConst& f, const float4* splats, const float* sh, float4* accum,
                          unsigned long long* stats, uint32_t* err, int sm_count, bool full, cudaStream_t st,
                          std::string* what);
cudaError_t sorted_read(SortedState& s, uint32_t* keys, uint32_t* vals, uint32_t n, cudaStream_t st);

}  // namespace gpsb
