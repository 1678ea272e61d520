// prim3.h -- launcher of k_prim3, the primitive kernel of the classes with generated VRR code.
#pragma once
#include <cuda_runtime.h>
#include "kernels.h"

namespace gint {

// The generated classes are instantiated in kPrim3Parts translation units (prim3.cu compiled
// with PRIM3_PART = 0..kPrim3Parts-1) so that they compile in parallel.
constexpr int kPrim3Parts = 8;

// Launches k_prim3 for class bt.cls if that class has generated code; returns false (and
// launches nothing) otherwise. *err receives the launch status.
bool prim3_launch(const DevCtx &ctx, const BatchArgs &bt, cudaStream_t st, cudaError_t *err);

// Loads every k_prim3 kernel and raises its shared-memory limit to smax bytes (see
// preload_kernels in kernels.h).
cudaError_t prim3_preload(int smax);

// one per part (prim3.cu)
bool prim3_launch_part0(const DevCtx &ctx, const BatchArgs &bt, cudaStream_t st, cudaError_t *err);
bool prim3_launch_part1(const DevCtx &ctx, const BatchArgs &bt, cudaStream_t st, cudaError_t *err);
bool prim3_launch_part2(const DevCtx &ctx, const BatchArgs &bt, cudaStream_t st, cudaError_t *err);
bool prim3_launch_part3(const DevCtx &ctx, const BatchArgs &bt, cudaStream_t st, cudaError_t *err);
bool prim3_launch_part4(const DevCtx &ctx, const BatchArgs &bt, cudaStream_t st, cudaError_t *err);
bool prim3_launch_part5(const DevCtx &ctx, const BatchArgs &bt, cudaStream_t st, cudaError_t *err);
bool prim3_launch_part6(const DevCtx &ctx, const BatchArgs &bt, cudaStream_t st, cudaError_t *err);
bool prim3_launch_part7(const DevCtx &ctx, const BatchArgs &bt, cudaStream_t st, cudaError_t *err);
cudaError_t prim3_preload_part0(int smax);
cudaError_t prim3_preload_part1(int smax);
cudaError_t prim3_preload_part2(int smax);
cudaError_t prim3_preload_part3(int smax);
cudaError_t prim3_preload_part4(int smax);
cudaError_t prim3_preload_part5(int smax);
cudaError_t prim3_preload_part6(int smax);
cudaError_t prim3_preload_part7(int smax);

}  // namespace gint
