// ref_cuda_harness.cu -- C entry points around the reference's UNMODIFIED
// CUDA path (src/cuda/CudaSimulation.cu and what it links).
//
// TEST INFRASTRUCTURE ONLY: the existing-GPU-kernel comparison.  oracle/
// Makefile compiles this file with the reference's own
// src/cuda/{DeviceBodies,CudaCollision,CudaQuadTree,CudaSimulation}.cu and
// src/Utils.cpp (read in place, never copied) for sm_100a into
// oracle/_ref/libref_cuda.so.  Every call lands in the reference's code:
// CudaSimulation(initial), its public dt/theta/epsilon/collisions
// (CudaSimulation.cuh:39-42) and step() (CudaSimulation.cu:51-58), timed
// as MainCuda.cu:121-184 does (CUDA events on the default stream around the
// step loop).  The reference aborts the process on any CUDA error
// (CUDA_CHECK, DeviceBodies.cuh:18-27), so callers run it in a child
// process.
#include "CudaSimulation.cuh"

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <vector>

static_assert(sizeof(Body) == 36, "Body is 36 bytes");

extern "C" {

// `warmup` untimed then `steps` timed CudaSimulation::step() calls on the
// given state; writes the final state back (device array order) and
// returns the milliseconds of the timed steps (CUDA events, default stream).
double ref_cuda_simulate(std::size_t n, Body *b, float dt, float theta,
                         float eps, int collisions, int warmup, int steps) {
  std::vector<Body> initial(b, b + n);
  CudaSimulation sim(initial);
  sim.dt = dt;
  sim.theta = theta;
  sim.epsilon = eps;
  sim.collisions = collisions != 0;
  for (int k = 0; k < warmup; ++k) sim.step();
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaDeviceSynchronize();
  cudaEventRecord(e0);
  for (int k = 0; k < steps; ++k) sim.step();
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  std::vector<Body> out;
  sim.bodies.download(out);
  std::memcpy(b, out.data(), n * sizeof(Body));
  return cudaGetLastError() == cudaSuccess ? (double)ms : -1.0;
}

} // extern "C"
