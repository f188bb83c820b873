// Hand-written build configuration for compiling the ScalFMM reference headers in place.
// It stands in for the CMake-generated header (the reference's Src/ScalFmmConfig.h.cmake) with the
// options of the reference's default CMake configuration: BLAS on, asserts on, the 256-bit AVX P2P
// (the fork's SCALFMM_USE_AVX2 branch is AVX-512, which not every host has), no MPI/StarPU/CUDA.
// FFT on: FFTW is not in this image, so oracle/ref/fftw supplies the FFTW 3 calls that FDft.hpp makes,
// as direct-summation DFTs, for the reference's Lagrange (uniform) kernel.
#ifndef SSCALFMMCONFIG_H
#define SSCALFMMCONFIG_H
#define SCALFMM_USE_BLAS
#define SCALFMM_USE_ASSERT
#define SCALFMM_USE_AVX
#define SCALFMM_USE_FFT
#include <string>
const std::string SCALFMMDataPath("./Data/");
const std::string SCALFMMCompileFlags("-O3 -fopenmp");
const std::string SCALFMMCompileLibs("openblas");
#endif
