// Host interface of the NVRTC specialization of k_step (aq_jit.cu).
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "../../include/aq.h"

namespace aq {

bool jit_available();
// Compile (or fetch from the in-process cache) k_step<D, HF, HM, R, JitLayout>
// for layout L; returns a CUfunction, or null with *err set.
void* jit_k_step(int D, bool HF, bool HM, bool f64, bool col, const aq_layout& L, std::string* err);
std::string jit_layout_source(const aq_layout& L);
int jit_set_smem(void* fn, int bytes);
int jit_occupancy(void* fn, int block, size_t smem, int* out);
int jit_launch(void* fn, unsigned grid, unsigned block, size_t smem, cudaStream_t st, void** args);

}  // namespace aq
