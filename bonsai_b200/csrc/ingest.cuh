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
    // a request plane (bb_plane_create_like): rows it was sized for, its
    // staging buffer and stream; 0 / null for planes made from one matrix
    uint64_t     cap_rows   = 0;
    float       *stage      = nullptr;
    uint64_t     stage_rows = 0;
    cudaStream_t stream     = nullptr;
};

// owned_stage (optional): a device staging buffer of owned_rows rows the
// caller keeps (a request plane's): host X then goes up through it with no
// allocation, chunk after chunk on `stream`, without waiting.
void ingest(Plane &p, float const *X, bool x_on_device, cudaStream_t stream,
            float *owned_stage = nullptr, uint64_t owned_rows = 0);

// Fills p.mirror from the feature-major codes (allocating it).
void build_mirror(Plane &p, cudaStream_t stream);

// Rows of a request plane's staging buffer for batches of up to max_rows:
// at most 64 MB, and a whole number of bin-application tiles whenever a batch
// can take more than one chunk.
uint64_t stage_rows_for(uint32_t n_feats, uint64_t max_rows);

// Rewrites p.mirror (already allocated for at least p.n_rows rows) from the
// feature-major codes.
void fill_mirror(Plane &p, cudaStream_t stream);

constexpr uint32_t k_mirror_bytes = 32;

} // namespace bb
