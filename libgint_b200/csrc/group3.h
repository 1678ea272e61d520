// group3.h -- launcher of k_group3, the per-lane group kernel of the classes with generated HRR.
#pragma once
#include <cuda_runtime.h>
#include "kernels.h"

namespace gint {

// The generated classes are instantiated in kGroup3Parts translation units (group3.cu compiled
// with GROUP3_PART = 0..kGroup3Parts-1) so that they compile in parallel.
constexpr int kGroup3Parts = 4;

// Launches k_group3 for class bt.cls if that class has generated code; returns false (and
// launches nothing) otherwise. *err receives the launch status.
bool group3_launch(const DevCtx &ctx, const BatchArgs &bt, cudaStream_t st, cudaError_t *err);

// Loads every k_group3 kernel (see preload_kernels in kernels.h).
cudaError_t group3_preload();

bool group3_launch_part0(const DevCtx &ctx, const BatchArgs &bt, cudaStream_t st, cudaError_t *err);
bool group3_launch_part1(const DevCtx &ctx, const BatchArgs &bt, cudaStream_t st, cudaError_t *err);
bool group3_launch_part2(const DevCtx &ctx, const BatchArgs &bt, cudaStream_t st, cudaError_t *err);
bool group3_launch_part3(const DevCtx &ctx, const BatchArgs &bt, cudaStream_t st, cudaError_t *err);
cudaError_t group3_preload_part0();
cudaError_t group3_preload_part1();
cudaError_t group3_preload_part2();
cudaError_t group3_preload_part3();

}  // namespace gint
