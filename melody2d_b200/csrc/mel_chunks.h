// Host builder of the Gauss-point chunk images read by the body kernel (layout in mel_internal.h).
#pragma once
#include <cstdint>
#include <vector>
#include "mel_internal.h"

struct mel_chunk_set {
    std::vector<mel_chunk> chunks;
    std::vector<int> b_chunk0;     // [n_bodies+1] first chunk of each body
    std::vector<uint8_t> img;      // all images, each 16-byte aligned
    int img_max = 16;              // largest image (bytes)
    long long n_entries = 0;       // stored entries, padding included
    long long n_pad = 0;           // padding entries (rounding of each chunk to 8 entries)
};

// Cuts every deformable body's Gauss points into chunks of at most MEL_CHUNK_GP_FP64 (FP64
// images) or MEL_CHUNK_GP_MX (FP32 images) points and at most `ecap` entries.  Returns MEL_OK or an error code with the message set.
// mixed: dN pairs stored as FP32 (the mixed-precision pass) instead of FP64.
mel_status mel_build_chunks(const mel_model_desc* d, int ecap, mel_chunk_set& out, bool mixed = false);
