// Grid dimensions and acoustic parameters as the kernels receive them (GridDims,
// timestep.js:88-90; AcousticParamsGPU, timestep.js:46-52), and the halo-3 field index
// (grid.js:181-199).  Plain C++: also compiled for the host.
#pragma once

#ifdef __CUDACC__
#define TE_HD_IDX __host__ __device__ __forceinline__
#else
#define TE_HD_IDX inline
#endif

namespace te {

struct Dims {
  int nx, ny, nz, sJ, sK;
  float rdx, rdy, rdz;
};

struct Acoustic {
  float dts, alph, beta, kdiv, smeps;
};

TE_HD_IDX int gidx(const Dims& g, int i, int j, int k) { return (i + 3) + g.sJ * ((j + 3) + g.sK * k); }

}  // namespace te
