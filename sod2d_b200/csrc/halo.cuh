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

// W > 0: the exchange width as a compile-time constant (the loops over the
// components unroll, so their loads are issued together); W = 0: v.width at
// run time.
template <class T, int W>
__global__ void k_halo_pack(int nsend, const int *__restrict__ node, HaloViewT<T> v, T *__restrict__ buf) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nsend) return;
  constexpr int MW = W > 0 ? W : HALO_MAX_WIDTH;
  const int width = W > 0 ? W : v.width;
  const long long p = (long long)node[j] * v.nstride;
  T val[MW];
#pragma unroll
  for (int k = 0; k < MW; ++k)
    if (k < width) val[k] = v.comp[k][p];
#pragma unroll
  for (int k = 0; k < MW; ++k)
    if (k < width) buf[(long long)j * width + k] = val[k];
}

// For shared node u: contributions ptr[u]..ptr[u+1]-1 in ascending rank
// order; src < 0 is this rank's own value, else a position in recv.
template <class T, int W>
__global__ void k_halo_sum(int nuniq, const int *__restrict__ uniq_node, const int *__restrict__ ptr,
                           const int *__restrict__ src, HaloViewT<T> v, const T *__restrict__ recv) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= nuniq) return;
  constexpr int MW = W > 0 ? W : HALO_MAX_WIDTH;
  const int width = W > 0 ? W : v.width;
  const long long p = (long long)uniq_node[u] * v.nstride;
  const int b = ptr[u], e = ptr[u + 1];
  T own[MW], acc[MW];
#pragma unroll
  for (int k = 0; k < MW; ++k)
    if (k < width) own[k] = v.comp[k][p];
  for (int i = b; i < e; ++i) {
    const int s = src[i];
    T x[MW];
#pragma unroll
    for (int k = 0; k < MW; ++k)
      if (k < width) x[k] = s < 0 ? own[k] : recv[(long long)s * width + k];
#pragma unroll
    for (int k = 0; k < MW; ++k)
      if (k < width) acc[k] = i == b ? x[k] : acc[k] + x[k];
  }
#pragma unroll
  for (int k = 0; k < MW; ++k)
    if (k < width) v.comp[k][p] = acc[k];
}

}  // namespace
