// Host interface of the NVRTC specialization of k_step (aq_jit.cu).
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "../../include/aq.h"
#include "aq_step_config.h"

namespace aq {

bool jit_available();
// Compile (or fetch from the in-process cache) k_step<D, HF, HM, R, JitLayout,
// col, sparse> for layout L; returns a CUfunction, or null with *err set.
void* jit_k_step(int D, bool HF, bool HM, bool f64, bool col, bool sparse, const aq_layout& L, std::string* err);
std::string jit_layout_source(const aq_layout& L);

// Whether the layout-specialized k_step keeps a record's words in
// registers (short records) rather than in a shared-memory slot per thread.
constexpr int kJitRegRecordMaxWords = 8;
inline bool jit_reg_record(const aq_layout& L) { return L.n_words <= kJitRegRecordMaxWords; }
// CTAs per SM k_step's registers are budgeted for: 80 registers a thread
// with register records, 128 with shared-memory slots
constexpr int kJitRegRecordMinBlocks = 768 / AQ_CH, kJitSlotMinBlocks = 512 / AQ_CH;
int jit_set_smem(void* fn, int bytes);
int jit_occupancy(void* fn, int block, size_t smem, int* out);
int jit_launch(void* fn, unsigned grid, unsigned block, size_t smem, cudaStream_t st, void** args);

}  // namespace aq
