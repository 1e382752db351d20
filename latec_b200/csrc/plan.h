// Host-side plan object behind the opaque latec_plan handle.
#pragma once

#include <mutex>
#include <vector>

#include "latec_common.cuh"

struct latec_plan {
    int ndim = 0;
    int levels = 0;
    int anchor_stride = 0;
    int anchor_block = 0;
    uint32_t shape[LATEC_MAX_NDIM] = {0};
    uint64_t points = 0;
    std::vector<latec::StageDesc> stages;
    // device copy of `stages` for the many-tensor launches, made on first use
    // (per device) and freed with the plan
    std::mutex dev_mu;
    latec::StageDesc* dev_stages = nullptr;
    int dev_id = -1;
    ~latec_plan() {
        if (dev_stages) cudaFree(dev_stages);
    }
};

namespace latec {
using Plan = latec_plan;
int check_plan(const uint32_t* shape, int ndim, int levels, int anchor_stride, int anchor_block);
int build_plan(Plan& p, const uint32_t* shape, int ndim, int levels, int anchor_stride,
               int anchor_block);
}  // namespace latec
