// Host-side layout of a plan object, shared by the .cu files of libtcpmvp.so.
#pragma once

#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "tcp_device.cuh"
#include "tcp_internal.h"

namespace tcp {

struct DeviceSchedule {
    Schedule host;
    RingSchedule ring;  // k_ring's schedule (tile_bits = 0: the plan does not use it)
    tcpdev::DevSchedule dev{};
};

// Page-locked staging ring of a host apply whose caller's buffers are
// ordinary (pageable) memory: kStageSlots slots of kStageSlotBytes; slot use u
// goes to slot u % kStageSlots, and ev[slot] marks the end of its last DMA.
constexpr int kStageSlots = 4;
constexpr size_t kStageSlotBytes = size_t(32) << 20;

struct Staging {
    unsigned char *host = nullptr;
    cudaEvent_t ev[kStageSlots] = {};
    uint64_t uses = 0;
};

struct Workspace {
    void *x = nullptr;
    void *y = nullptr;
    size_t bytes = 0;
    Staging *stage = nullptr;  // allocated on the first pageable apply
};

int cuda_fail(cudaError_t e, const char *what);
cudaError_t dev_malloc(void **p, size_t bytes);

}  // namespace tcp

struct tcp_mvp_plan {
    uint32_t nqubits = 0;
    uint32_t word_count = 0;
    uint64_t dim = 0;
    int storage = 0;
    int device = 0;
    int64_t transitions = -1;
    std::vector<tcp::MatrixTerm> terms;
    uint64_t group_count = 0;
    tcp::DeviceSchedule sched;  // one schedule (4096-row tiles) serves both precisions
    void *dev_block = nullptr;
    size_t dev_bytes = 0;
    int *d_err = nullptr;
    mutable std::mutex ws_mutex;
    mutable std::vector<tcp::Workspace> ws_free;
    mutable std::vector<tcp::Workspace> ws_all;
};

namespace tcp {
int check_plan(const tcp_mvp_plan *plan);
int length_error(uint64_t expected, uint64_t actual);
bool overlaps(const void *a, const void *b, size_t bytes);
int ring_prepare(const tcp_mvp_plan *p, bool c64);
int launch_ring_rhs(const tcp_mvp_plan *p, const void *x, void *y, uint32_t nrhs, bool c64, int *err,
                    cudaStream_t stream);
}  // namespace tcp
