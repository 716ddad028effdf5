// A non-Python caller of the C-ABI, as the Fortran solver would be: it holds
// the mesh and the state in host arrays of the reference's Fortran layout
// (read here from flat little-endian files), builds the context with
// sod_gpu_init, moves the state to the device, calls sod_gpu_comp_tau and
// sod_gpu_updateF, and writes the residuals back to flat files.
//
//   abi_harness <dir>
//
// <dir>/sizes.txt: porder nelem npoin npoin_w; then the arrays named below
// as raw binary (int32 or float32).  Output: <dir>/Rmass.bin, Rmom.bin,
// Rener.bin (float32).  Exit status 0 on success.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#include "sod2d_gpu.h"

template <class T>
static std::vector<T> load(const std::string &path, size_t n) {
  std::vector<T> v(n);
  std::ifstream f(path, std::ios::binary);
  if (!f || !f.read(reinterpret_cast<char *>(v.data()), (std::streamsize)(n * sizeof(T)))) {
    std::fprintf(stderr, "cannot read %s\n", path.c_str());
    std::exit(2);
  }
  return v;
}

template <class T>
static void save(const std::string &path, const std::vector<T> &v) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char *>(v.data()), (std::streamsize)(v.size() * sizeof(T)));
}

static float *to_device(const std::vector<float> &h) {
  float *d = nullptr;
  if (cudaMalloc(&d, h.size() * sizeof(float)) != cudaSuccess ||
      cudaMemcpy(d, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
    std::fprintf(stderr, "device allocation failed\n");
    std::exit(3);
  }
  return d;
}

#define CHECK(call)                                                              \
  do {                                                                           \
    if ((call) != 0) {                                                           \
      std::fprintf(stderr, "%s failed: %s\n", #call, sod_gpu_last_error());      \
      return 1;                                                                  \
    }                                                                            \
  } while (0)

int main(int argc, char **argv) {
  if (argc != 2) {
    std::fprintf(stderr, "usage: %s <dir>\n", argv[0]);
    return 2;
  }
  const std::string dir = std::string(argv[1]) + "/";
  int porder = 0, nelem = 0, npoin = 0, npoin_w = 0;
  {
    std::ifstream s(dir + "sizes.txt");
    s >> porder >> nelem >> npoin >> npoin_w;
  }
  const size_t n1 = porder + 1, nnode = n1 * n1 * n1, ngaus = nnode;
  // mesh, reference layout (column-major, 1-based connectivity)
  auto connec = load<int>(dir + "connec.bin", (size_t)nelem * nnode);
  auto lpoin_w = load<int>(dir + "lpoin_w.bin", npoin_w);
  auto invA = load<int>(dir + "invAtoIJK.bin", n1 * n1 * n1);
  auto gI = load<int>(dir + "gmshAtoI.bin", nnode), gJ = load<int>(dir + "gmshAtoJ.bin", nnode),
       gK = load<int>(dir + "gmshAtoK.bin", nnode);
  auto dl = load<float>(dir + "dlxigp_ip.bin", ngaus * 3 * n1);
  auto He = load<float>(dir + "He.bin", 9 * ngaus * (size_t)nelem);
  auto gpvol = load<float>(dir + "gpvol.bin", ngaus * (size_t)nelem);
  auto Ml = load<float>(dir + "Ml.bin", npoin), invMl = load<float>(dir + "invMl.bin", npoin);
  auto helem = load<float>(dir + "helem.bin", nelem);
  auto helem_l = load<float>(dir + "helem_l.bin", (size_t)nelem * nnode);
  auto lelpn = load<int>(dir + "lelpn.bin", npoin);
  auto Ngp = load<float>(dir + "Ngp.bin", ngaus * nnode);
  auto phys_v = load<float>(dir + "phys.bin", 14);
  // state
  auto rho = load<float>(dir + "rho.bin", npoin), q = load<float>(dir + "q.bin", 3 * (size_t)npoin),
       E = load<float>(dir + "E.bin", npoin), u = load<float>(dir + "u.bin", 3 * (size_t)npoin),
       csound = load<float>(dir + "csound.bin", npoin),
       mu_e = load<float>(dir + "mu_e.bin", (size_t)nelem * ngaus);
  const float mu_factor = load<float>(dir + "mu_factor.bin", 1)[0];

  sod_mesh_t mesh{};
  mesh.porder = porder; mesh.nelem = nelem; mesh.npoin = npoin; mesh.npoin_w = npoin_w;
  mesh.connec = connec.data(); mesh.lpoin_w = lpoin_w.data(); mesh.invAtoIJK = invA.data();
  mesh.gmshAtoI = gI.data(); mesh.gmshAtoJ = gJ.data(); mesh.gmshAtoK = gK.data();
  mesh.dlxigp_ip = dl.data(); mesh.He = He.data(); mesh.gpvol = gpvol.data(); mesh.Ml = Ml.data();
  mesh.invMl = invMl.data(); mesh.helem = helem.data(); mesh.helem_l = helem_l.data();
  mesh.lelpn = lelpn.data(); mesh.Ngp = Ngp.data();
  sod_phys_t phys{};  // phys.bin holds the 14 constants in the declaration order
  phys.gamma_gas = phys_v[0]; phys.Rgas = phys_v[1]; phys.Cp = phys_v[2]; phys.Prt = phys_v[3];
  phys.c_lps = phys_v[4]; phys.c_rho = phys_v[5]; phys.c_ener = phys_v[6]; phys.ce = phys_v[7];
  phys.cmax = phys_v[8]; phys.cglob = phys_v[9]; phys.ducros_min_val = phys_v[10];
  phys.c_species_stab = phys_v[11]; phys.p_inf = phys_v[12]; phys.rho_inf = phys_v[13];

  sod_gpu_ctx *ctx = nullptr;
  CHECK(sod_gpu_init(&mesh, &phys, &ctx));
  float *d_rho = to_device(rho), *d_q = to_device(q), *d_E = to_device(E), *d_u = to_device(u),
        *d_c = to_device(csound), *d_mue = to_device(mu_e);
  std::vector<float> zeroN(npoin, 0.f), zero3N(3 * (size_t)npoin, 0.f), zeroE(nelem, 0.f);
  float *d_tau = to_device(zeroE), *d_Rm = to_device(zeroN), *d_Rq = to_device(zero3N), *d_Re = to_device(zeroN);
  CHECK(sod_gpu_comp_tau(ctx, d_c, d_u, d_tau));
  CHECK(sod_gpu_updateF(ctx, d_rho, d_q, d_E, d_mue, mu_factor, d_tau, d_Rm, d_Rq, d_Re, nullptr, nullptr,
                        nullptr, nullptr));
  std::vector<float> Rm(npoin), Rq(3 * (size_t)npoin), Re(npoin);
  cudaMemcpy(Rm.data(), d_Rm, Rm.size() * 4, cudaMemcpyDeviceToHost);
  cudaMemcpy(Rq.data(), d_Rq, Rq.size() * 4, cudaMemcpyDeviceToHost);
  cudaMemcpy(Re.data(), d_Re, Re.size() * 4, cudaMemcpyDeviceToHost);
  save(dir + "Rmass.bin", Rm);
  save(dir + "Rmom.bin", Rq);
  save(dir + "Rener.bin", Re);
  for (float *p : {d_rho, d_q, d_E, d_u, d_c, d_mue, d_tau, d_Rm, d_Rq, d_Re}) cudaFree(p);
  CHECK(sod_gpu_finalize(ctx));
  std::printf("abi harness ok: %d elements, %d nodes\n", nelem, npoin);
  return 0;
}
