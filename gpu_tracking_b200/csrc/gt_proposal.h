// gt_proposal.h — the learned proposal network object behind the C ABI's
// gt_proposal handle (device parameters, Adam state, packed UMMA operands).
#pragma once

#include "gt_kernels.h"

struct gt_proposal {
    int device = 0;
    float mean = 0.0f;       // input normalisation: (pixel - mean) * scale
    float scale = 1.0f;
    float threshold = 0.0f;  // score logit a cell must exceed to propose a seed
    float* params = nullptr;  // fp32 master copy, kCnnParams
    float* adam_m = nullptr;
    float* adam_v = nullptr;
    float* grad = nullptr;
    int64_t adam_t = 0;
    uint8_t* packed = nullptr;  // BF16 operands: forward layers 0-3, backward layers 1-3
    size_t off_f[gt::kCnnLayers] = {};
    size_t off_d[gt::kCnnLayers] = {};
    size_t packed_bytes = 0;

    gt::CnnNet views() const {
        gt::CnnNet n;
        for (int l = 0; l < gt::kCnnLayers; l++) {
            n.wf[l] = packed + off_f[l];
            n.wd[l] = l > 0 ? packed + off_d[l] : nullptr;
            n.bias[l] = params + gt::cnn_layer_offset(l) + gt::kCnnCout[l] * gt::kCnnCin[l] * 9;
        }
        return n;
    }
};

namespace gt {
// Rebuild the packed BF16 operands from the fp32 parameters.
cudaError_t proposal_repack(const gt_proposal* p, cudaStream_t st);
}  // namespace gt
