/*
 * Launchers for STIR's own CUDA prior kernels (cut out of the STIR tree into oracle/_ref/cuda_priors_extracted.cuh by
 * extract_cuda_priors.py) with the launch configuration of STIR's host classes, on device-resident images: the
 * reference's sm_100 build, timed and compared against the B200 Gibbs kernels on the same box.  Test and benchmark
 * infrastructure only.
 *
 *   CudaRelativeDifferencePrior::compute_gradient (CudaRelativeDifferencePrior.cu:240-300): blocks of 8x8x8 threads
 *     over (x, y, z), the 3x3x3 weights on the device;
 *   CudaGibbsPenalty::compute_gradient (CudaGibbsPenalty.cuh:500-543, set-up :676-700): blocks of 8x8x1, the
 *     image and weight index ranges as int3 in the order the set-up fills them.
 * Images are [z][y][x] (STIR's order); no host copies.
 */
#include "cuda_priors_extracted.cuh"

extern "C" int ref_cuda_rdp_prior_gradient(float* grad, const float* image, const float* weights27, const float* kappa,
                                           float gamma, float epsilon, float penalisation_factor, int nz, int ny,
                                           int nx, void* stream) {
  const dim3 block(8, 8, 8);
  const dim3 grid((nx + 7) / 8, (ny + 7) / 8, (nz + 7) / 8);
  stir::computeCudaRelativeDifferencePriorGradientKernel<float><<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(
      grad, image, weights27, kappa, kappa != nullptr, gamma, epsilon, penalisation_factor, nz, ny, nx);
  return static_cast<int>(cudaGetLastError());
}

/* potential: 0 quadratic, 1 relative difference.  weights [z][y][x] of sizes wz x wy x wx on the device, index
   ranges -(size/2) .. size-1-size/2; the image index ranges z 0..nz-1, y min_y.., x min_x.. */
extern "C" int ref_cuda_gibbs_gradient(int potential, float* grad, const float* image, const float* weights, int wz,
                                       int wy, int wx, const float* kappa, float penalisation_factor, float gamma,
                                       float epsilon, int nz, int ny, int nx, int min_y, int min_x, void* stream) {
  const int3 dim = make_int3(nx, ny, nz);
  const int3 img_min = make_int3(min_x, min_y, 0);
  const int3 img_max = make_int3(min_x + nx - 1, min_y + ny - 1, nz - 1);
  // (weights.get_max_index(), weights[0].get_max_index(), weights[0][0].get_max_index()): z, y, x
  const int3 w_min = make_int3(-(wz / 2), -(wy / 2), -(wx / 2));
  const int3 w_max = make_int3(wz - 1 - wz / 2, wy - 1 - wy / 2, wx - 1 - wx / 2);
  const dim3 block(8, 8, 1);
  const dim3 grid((nx + 7) / 8, (ny + 7) / 8, nz);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (potential == 1) {
    stir::RelativeDifferencePotential<float> pot;
    pot.gamma = gamma;
    pot.epsilon = epsilon;
    stir::CudaGibbsPenalty_gradient_kernel<float, stir::RelativeDifferencePotential<float>><<<grid, block, 0, st>>>(
        grad, image, weights, kappa, kappa != nullptr, penalisation_factor, dim, img_max, img_min, w_max, w_min, pot);
  } else {
    stir::QuadraticPotential<float> pot;
    stir::CudaGibbsPenalty_gradient_kernel<float, stir::QuadraticPotential<float>><<<grid, block, 0, st>>>(
        grad, image, weights, kappa, kappa != nullptr, penalisation_factor, dim, img_max, img_min, w_max, w_min, pot);
  }
  return static_cast<int>(cudaGetLastError());
}
