// Halo sum of assembled nodal fields across the ranks of a partitioned mesh:
// the counterpart of mpi_halo_atomic_update_real_arrays /
// mpi_halo_atomic_update_real_massEnerMom with the NCCL transport
// (src/lib_sod2d/sources/mod_comms.f90:776-877, :1049-1102, :1795-1822).
//
// The reference packs the shared nodes of each neighbour into a send buffer
// (fill_sendBuffer_*, mod_comms.f90:431-520), exchanges the buffers with
// ncclSend/ncclRecv and adds what it received with atomics, neighbour by
// neighbour (copy_from_rcvBuffer_*).  A node shared by three or more ranks
// is then summed in a different order on each rank, so the ranks can end up
// with values that differ in the last bit.  Here every shared node is summed
// over its ranks in ascending rank order, its own value taking its rank's
// place, so all ranks hold bit-identical values afterwards.
//
// Buffers follow the reference: for node j of the concatenated list
// nodesToComm (neighbour ranges in ranksToComm order) and component k of a
// width-W exchange, the value sits at j*W + k.
#pragma once

#include <cuda_runtime.h>

namespace {

constexpr int HALO_MAX_WIDTH = 12;

// Component k of node p is comp[k][p * nstride]: a node-major buffer of
// width W (comp[k] = base + k, nstride = W) or reference-layout (npoin,ncomp)
// arrays (comp[k] = base + k*npoin, nstride = 1).  T is float, or double for
// the FP64 pressure solve (a double travels as two floats of the buffers).
template <class T>
struct HaloViewT {
  T *comp[HALO_MAX_WIDTH];
  int width;
  long long nstride;
};
using HaloView = HaloViewT<float>;

template <class T>
__global__ void k_halo_pack(int nsend, const int *__restrict__ node, HaloViewT<T> v, T *__restrict__ buf) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nsend) return;
  const long long p = (long long)node[j] * v.nstride;
  T val[HALO_MAX_WIDTH];
#pragma unroll
  for (int k = 0; k < HALO_MAX_WIDTH; ++k)
    if (k < v.width) val[k] = v.comp[k][p];
#pragma unroll
  for (int k = 0; k < HALO_MAX_WIDTH; ++k)
    if (k < v.width) buf[(long long)j * v.width + k] = val[k];
}

// For shared node u: contributions ptr[u]..ptr[u+1]-1 in ascending rank
// order; src < 0 is this rank's own value, else a position in recv.
template <class T>
__global__ void k_halo_sum(int nuniq, const int *__restrict__ uniq_node, const int *__restrict__ ptr,
                           const int *__restrict__ src, HaloViewT<T> v, const T *__restrict__ recv) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= nuniq) return;
  const long long p = (long long)uniq_node[u] * v.nstride;
  const int b = ptr[u], e = ptr[u + 1];
  for (int k = 0; k < v.width; ++k) {
    const T own = v.comp[k][p];
    T acc = 0;
    for (int i = b; i < e; ++i) {
      const int s = src[i];
      const T x = s < 0 ? own : recv[(long long)s * v.width + k];
      acc = i == b ? x : acc + x;
    }
    v.comp[k][p] = acc;
  }
}

}  // namespace
