// Bin application: raw row-major float32 features -> feature-major bin codes.
//
// Restates BinMapper::transform (src/bin_mapper.cpp:284-291): a value's bin
// is the number of cuts strictly below it (lower_bound), and NaN takes the
// last bin. The reference's device twin is transform_bin in
// src/cuda/detail/ingest_kernels.cuh:28-50, one scalar thread per cell; this
// kernel instead stages a (rows x features) tile of X through shared memory
// with 16-byte loads and writes each feature's run of 16 (u8) or 8 (u16)
// consecutive rows as one 16-byte store.
#pragma once

#include "common.cuh"

namespace bb
{

// One device-resident binned dataset. Bins are feature-major:
// bins[f * n_pad + r], n_pad a multiple of 64 so every column starts on a
// 64-byte boundary and 16-byte vector loads/stores line up.
struct Plane
{
    uint64_t  n_rows   = 0;
    uint64_t  n_pad    = 0;
    uint32_t  n_feats  = 0;
    bool      u8       = true;
    void     *bins     = nullptr; // uint8_t or uint16_t
    // Row-major mirror for gathered reads: features in tiles of 32 bytes
    // (32 u8 or 16 u16 codes), tile t of row r at mirror[(t * n_rows + r) * 32],
    // so one gathered row costs one 32-byte DRAM sector per tile.
    void     *mirror   = nullptr;
    uint32_t  n_tiles  = 0;
    float    *cuts     = nullptr; // flattened cuts, device
    uint32_t *cut_off  = nullptr; // F + 1 offsets, device
    uint32_t *n_bins   = nullptr; // per feature, device
    int       device   = 0;
    // host copies of the mapper tables
    float    *h_cuts    = nullptr;
    uint32_t *h_cut_off = nullptr;
};

void ingest(Plane &p, float const *X, bool x_on_device, cudaStream_t stream);

// Fills p.mirror from the feature-major codes (allocating it).
void build_mirror(Plane &p, cudaStream_t stream);

constexpr uint32_t k_mirror_bytes = 32;

} // namespace bb
