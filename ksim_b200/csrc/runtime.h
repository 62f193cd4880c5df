// runtime.h — host-side objects behind the C ABI handles.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ksim_b200.h"
#include "image.h"
#include "kernels.h"

namespace ksim {

ksim_status fail(ksim_status s, const std::string &m);
ksim_status cuda_fail(cudaError_t e, const char *what);

// Select a device for the lifetime of a call and restore the caller's.
struct DeviceGuard {
    int prev = -1;
    bool ok = true;
    explicit DeviceGuard(int dev);
    ~DeviceGuard();
};

// Grow-only device workspace.
struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t n);
    void release();
};

struct ComponentChunks {
    ChunkDir *d = nullptr;
    int n = 0;
};

}  // namespace ksim

struct ksim_component {
    int device = 0;
    ksim::HostImage img;  // directory and term offsets (packed bytes freed after upload)
    uint8_t *d_image = nullptr;
    size_t image_bytes = 0;
    std::map<int, ksim::ComponentChunks> chunks;  // by staging slot size
    uint32_t *d_status = nullptr;
    cudaStream_t stream = nullptr;
    ksim::DevBuf ws_f, ws_out, ws_aux;
    ksim::LaunchCfg cfg;
    int64_t wait_limit = 0;  // polls of a staging wait (0: the kernels' default)
    ksim_program *self_prog = nullptr;  // this component alone as a program (host-buffer sample calls)
    std::mutex mu;        // workspaces, cfg and self_prog
    std::mutex chunk_mu;  // the chunk-directory map
};

struct ProgramPart {
    ksim_component *comp = nullptr;
    int32_t *d_sel = nullptr;   // f_selection on the device
    int32_t *d_cols = nullptr;  // destination output column of each component output
};

#ifndef KSIM_HOST_STREAMS
#define KSIM_HOST_STREAMS 4
#endif

struct ksim_program {
    int device = 0;
    int n_outputs = 0;
    int min_f_cols = 0;
    std::vector<ProgramPart> parts;
    // host-buffer calls: KSIM_HOST_STREAMS compute streams taken in turn
    // (consecutive chunks overlap) and one stream per copy direction
    cudaStream_t cs[KSIM_HOST_STREAMS] = {}, s_h2d = nullptr, s_d2h = nullptr;
    std::vector<cudaEvent_t> ev_in, ev_done;  // per chunk, kept across calls
    uint32_t *h_status = nullptr;             // page-locked: the components' status words after a call
    int64_t wave_shots = 1;                   // shots one wave of sampling CTAs holds on the device
    ksim::DevBuf ws_f, ws_out, ws_fp, ws_op;  // unpacked rows; bit-packed rows
    std::mutex mu;
};

namespace ksim {
ksim_status component_chunks(ksim_component *c, int slot_bytes, const ChunkDir **d, int *n);
ksim_status component_job(ksim_component *c, const LaunchCfg &cfg, SampleJob &j);
}  // namespace ksim
