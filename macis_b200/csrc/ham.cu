// Hamiltonian generator state in HBM: integrals and the intermediates of
// HamiltonianGenerator::generate_integral_intermediates
// (include/macis/hamiltonian_generator/impl.hpp:26-70), plus the batched
// matrix_element entry point (hamiltonian_generator/matrix_elements.hpp:15).
#include "internal.hpp"
#include "primitives.cuh"

namespace mb {

// G(i,j,k,l) = V(i,j,k,l) - V(i,l,k,j)  (impl.hpp:36-43)
__global__ void g_from_v_k(const double* __restrict__ V, double* __restrict__ G,
                           int n) {
  const size_t n4 = size_t(n) * n * n * n;
  for(size_t x = size_t(blockIdx.x) * blockDim.x + threadIdx.x; x < n4;
      x += size_t(gridDim.x) * blockDim.x) {
    const size_t i = x % n, j = (x / n) % n, k = (x / n / n) % n,
                 l = x / n / n / n;
    G[x] = V[x] - V[idx4(int(i), int(l), int(k), int(j), n)];
  }
}

// G_red(k,i,j) = G(k,k,i,j), V_red(k,i,j) = V(k,k,i,j)  (impl.hpp:45-56)
// G2_red(i,j) = 0.5 G(i,i,j,j), V2_red(i,j) = V(i,i,j,j)  (impl.hpp:58-68)
__global__ void reduced_k(const double* __restrict__ V,
                          const double* __restrict__ G, double* G_red,
                          double* V_red, double* G2_red, double* V2_red,
                          int n) {
  const size_t n3 = size_t(n) * n * n;
  for(size_t x = size_t(blockIdx.x) * blockDim.x + threadIdx.x; x < n3;
      x += size_t(gridDim.x) * blockDim.x) {
    const int k = int(x % n), i = int((x / n) % n), j = int(x / n / n);
    G_red[x] = G[idx4(k, k, i, j, n)];
    V_red[x] = V[idx4(k, k, i, j, n)];
    if(k == 0) {
      G2_red[i + size_t(j) * n] = 0.5 * G[idx4(i, i, j, j, n)];
      V2_red[i + size_t(j) * n] = V[idx4(i, i, j, j, n)];
    }
  }
}

template <int NBITS>
__global__ void matel_k(Ints I, const uint64_t* bra, const uint64_t* ket,
                        size_t n, double* out) {
  using D = DetTraits<NBITS>;
  for(size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
      i += size_t(gridDim.x) * blockDim.x) {
    const uint64_t* b = bra + i * D::NW;
    const uint64_t* k = ket + i * D::NW;
    out[i] = me_generic(I, D::alpha(b), D::beta(b), D::alpha(k), D::beta(k));
  }
}

void matrix_elements_device(macis_b200_ham* h, const uint64_t* bra,
                            const uint64_t* ket, size_t n, double* out) {
  if(!n) return;
  const unsigned g = grid_for(n, 128, 16 * num_sms());
  auto I = h->ints();
  if(h->nbits == 64)
    matel_k<64><<<g, 128, 0, h->stream>>>(I, bra, ket, n, out), note_launch();
  else if(h->nbits == 128)
    matel_k<128><<<g, 128, 0, h->stream>>>(I, bra, ket, n, out), note_launch();
  else
    matel_k<256><<<g, 128, 0, h->stream>>>(I, bra, ket, n, out), note_launch();
  MB_CUDA(cudaGetLastError());
}

void ham_create(macis_b200_ham* h, int nbits, size_t norb, const double* T,
                size_t LDT, const double* V, size_t LDV) {
  MB_REQUIRE(nbits == 64 || nbits == 128 || nbits == 256, MACIS_B200_EINVAL,
             "nbits must be 64, 128 or 256");
  MB_REQUIRE(norb >= 1 && 2 * norb <= size_t(nbits) && norb <= 127,
             MACIS_B200_EINVAL, "norb must satisfy 1 <= norb <= nbits/2");
  MB_REQUIRE(LDT >= norb && LDV >= norb, MACIS_B200_EINVAL,
             "leading dimension smaller than norb");
  const size_t n = norb, n2 = n * n, n3 = n2 * n, n4 = n3 * n;
  h->nbits = nbits;
  h->norb = int(norb);
  MB_CUDA(cudaGetDevice(&h->device));
  MB_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  // keep freed stream-ordered allocations cached in this process (CSR and
  // scratch buffers are reused across builds)
  cudaMemPool_t pool;
  MB_CUDA(cudaDeviceGetDefaultMemPool(&pool, h->device));
  uint64_t thr = ~0ull;
  MB_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
  // Pack to compact leading dimensions on the host.
  std::vector<double> t(n2), v(n4);
  for(size_t q = 0; q < n; ++q)
    for(size_t p = 0; p < n; ++p) t[p + q * n] = T[p + q * LDT];
  for(size_t s = 0; s < n; ++s)
    for(size_t r = 0; r < n; ++r)
      for(size_t q = 0; q < n; ++q)
        for(size_t p = 0; p < n; ++p)
          v[p + n * (q + n * (r + n * s))] = V[p + LDV * (q + LDV * (r + LDV * s))];
  MB_CUDA(dev_malloc(&h->T, n2 * 8));
  MB_CUDA(dev_malloc(&h->V, n4 * 8));
  MB_CUDA(dev_malloc(&h->G, n4 * 8));
  MB_CUDA(dev_malloc(&h->G_red, n3 * 8));
  MB_CUDA(dev_malloc(&h->V_red, n3 * 8));
  MB_CUDA(dev_malloc(&h->G2_red, n2 * 8));
  MB_CUDA(dev_malloc(&h->V2_red, n2 * 8));
  MB_CUDA(cudaMemcpyAsync(h->T, t.data(), n2 * 8, cudaMemcpyHostToDevice, h->stream));
  MB_CUDA(cudaMemcpyAsync(h->V, v.data(), n4 * 8, cudaMemcpyHostToDevice, h->stream));
  g_from_v_k<<<grid_for(n4, 256, 8 * num_sms()), 256, 0, h->stream>>>(h->V, h->G, int(n)), note_launch();
  reduced_k<<<grid_for(n3, 256, 8 * num_sms()), 256, 0, h->stream>>>(
      h->V, h->G, h->G_red, h->V_red, h->G2_red, h->V2_red, int(n)), note_launch();
  MB_CUDA(cudaGetLastError());
  MB_CUDA(cudaStreamSynchronize(h->stream));
}

void ham_destroy(macis_b200_ham* h) {
  if(!h) return;
  cudaFree(h->T);
  cudaFree(h->V);
  cudaFree(h->G);
  cudaFree(h->G_red);
  cudaFree(h->V_red);
  cudaFree(h->G2_red);
  cudaFree(h->V2_red);
  cudaFree(h->VT);
  cudaFree(h->pairmax);
  if(h->stream) cudaStreamDestroy(h->stream);
}

}  // namespace mb
