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
    std::vector<int> b_pipe;       // [n_bodies] 1: the body runs the three-stage pipeline (mixed only)
};

// Cuts every deformable body's Gauss points into chunks of at most `ecap` entries and at most
// MEL_CHUNK_GP_FP64 points, or MEL_CHUNK_GP_MX points for a body that runs the mixed pass's
// three-stage pipeline (its point threads are fewer).  mixed: dN pairs stored as FP32 instead of
// FP64; a mixed body runs the pipeline when it has at least pipe_min_entries support entries
// (out.b_pipe).  Returns MEL_OK or an error code with the message set.
mel_status mel_build_chunks(const mel_model_desc* d, int ecap, mel_chunk_set& out, bool mixed = false,
                            long long pipe_min_entries = 0);
// support entries of deformable body b
long long mel_body_entries(const mel_model_desc* d, int b);
