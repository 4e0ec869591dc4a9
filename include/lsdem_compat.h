/*
 * lsdem_compat — the reference solver's separable extern "C" launchers, with its
 * own signatures, implemented by liblsdem_b200 on this library's kernels. For host
 * code written against the reference's internal launcher layer (its own LSSolver
 * and helper classes call these); applications use the C ABI (lsdem_b200.h) or the
 * drop-in LSSolver (kernel/LSSolver.h) instead.
 *
 * Device pointers are the caller's; every launcher is asynchronous on `stream` and,
 * as in the reference, returns nothing: errors surface through cudaGetLastError.
 * The grid and block sizes the reference takes are accepted and not used.
 * Paths are relative to the reference project root.
 */
#ifndef LSDEM_COMPAT_H
#define LSDEM_COMPAT_H

#include <cuda_runtime.h>
#include <stddef.h>

#include "kernel/CUDAKernelFunction/myUtility/myMat.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Cell key of every object (-1 outside [minBound, maxBound)), then a stable sort by key:
 * hashValue holds the sorted keys, hashIndex the sorted object indices, gridHashStart /
 * gridHashEnd the [start, end) of every cell in the sorted order (-1 when empty; keys
 * outside [0, numGrid) belong to no cell). Replaces launchUpdateSpatialGridHashStartEnd
 * (FunDEM/kernel/CUDAKernelFunction/myUtility/mySpatialGrid.h:33-49,
 * mySpatialGrid.cu:242-277, buildHashStartEnd.cu:69-137). Its scratch (keys and sort
 * buckets) is allocated by the library on first use and kept, grown as needed. */
void launchUpdateSpatialGridHashStartEnd(int* hashIndex, int* hashValue, const double3* position, int* gridHashStart,
                                         int* gridHashEnd, const double3 minBound, const double3 maxBound,
                                         const double3 inverseCellSize, const int3 gridSize3D, const size_t numGrid,
                                         const size_t numObject, const size_t gridD_GPU, const size_t blockD_GPU,
                                         cudaStream_t stream_GPU);

/* velocity += (force invMass + gravity) timeStep and angularVelocity += (R invI R^T)
 * torque timeStep for every object with invMass != 0. Replaces
 * launchParticleVelocityAngularVelocityIntegration
 * (FunDEM/kernel/CUDAKernelFunction/particleIntegrationKernel.cuh:4-17,
 * particleIntegrationKernel.cu:3-22). */
void launchParticleVelocityAngularVelocityIntegration(double3* velocity, double3* angularVelocity,
                                                      const double3* force, const double3* torque,
                                                      const double* invMass, const quaternion* orientation,
                                                      const symMatrix* inverseInertiaTensor, const double3 gravity,
                                                      const double timeStep, const size_t num, const size_t gridD,
                                                      const size_t blockD, cudaStream_t stream);

/* position += timeStep velocity; orientation integrated with angularVelocity over
 * timeStep and normalised. Replaces launchParticlePositionOrientationIntegration
 * (particleIntegrationKernel.cuh:19-30, particleIntegrationKernel.cu:24-40). */
void launchParticlePositionOrientationIntegration(double3* position, quaternion* orientation, const double3* velocity,
                                                  const double3* angularVelocity, const double timeStep,
                                                  const size_t num, const size_t gridD, const size_t blockD,
                                                  cudaStream_t stream);

/* Periodic wrap along x / y: a coordinate below the minimum gains, one at or above the
 * maximum loses, the domain length. Replaces launchUpdatePositionOutOfBoundaryXD / YD
 * (FunDEM/kernel/CUDAKernelFunction/myUtility/mySpatialGrid.h:51-65, mySpatialGrid.cu:28-56). */
void launchUpdatePositionOutOfBoundaryXD(double3* position, const double3 minBound, const double3 maxBound,
                                         const size_t numObject, const size_t gridD, const size_t blockD,
                                         cudaStream_t stream);
void launchUpdatePositionOutOfBoundaryYD(double3* position, const double3 minBound, const double3 maxBound,
                                         const size_t numObject, const size_t gridD, const size_t blockD,
                                         cudaStream_t stream);

#ifdef __cplusplus
}
#endif
#endif
