// rh_io.cu — restart (backup) and snapshot (output) file images of the hydro
// state in the reference's byte layouts (include/ramses_hydro_io.h), built in
// device memory from the resident state.
//
//   amr file    amr/output_amr.f90:607-660 output_amr, :666-735 backup_amr
//   hydro file  hydro/output_hydro.f90:167-246 backup_hydro (float64 uold),
//               hydro/output_hydro.f90:40-162 output_hydro (float32 primitives)
//   headers     amr/ramses_commons.f90:138-158 open_file, and the header
//               writes of backup_amr / backup_hydro (identical layouts)
//
// The hydro payload is the heavy part (320 B per oct for a backup): it is made
// by one bandwidth-bound kernel (or one device copy, for an FP64 backup) per
// level straight from the state buffers into the image, which then leaves the
// device in one copy.  The amr payload (16 B per oct) comes from the host's
// oct records.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "ramses_hydro_io.h"
#include "rh_internal.h"

namespace rh {

namespace {

void* g_image = nullptr;  // library-owned image (device), grown on demand
size_t g_image_cap = 0;

int ensure_image(size_t bytes) {
  if (bytes <= g_image_cap) return RH_OK;
  Context& c = ctx();
  RH_CUDA(cudaStreamSynchronize(c.stream));
  cudaFree(g_image);
  g_image = nullptr;
  g_image_cap = 0;
  const size_t cap = std::max(bytes + bytes / 8, (size_t)1 << 20);
  RH_CUDA(cudaMalloc(&g_image, cap));
  g_image_cap = cap;
  return RH_OK;
}

// output_hydro (hydro/output_hydro.f90:86-140, hydro only: no MHD field, no
// non-thermal energies, no passive scalars): rho, u = (rho u)/rho, v, w and
// p = (gamma-1)(E - ekin), ekin = 0.5 rho (u*u + v*v + w*w), each operation
// rounded as written (no contraction), then rounded to float32
// (real(qold, kind=4)).  One thread per cell; the image keeps the per-oct
// q(1:8, 1:5) order.
__global__ void prim_image_kernel(const double* __restrict__ ud, const float* __restrict__ uf, int bulk,
                                  long long noct, double gm1, uint32_t* __restrict__ dst) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= noct * 8) return;
  const long long o = i >> 3;
  const int cell = (int)(i & 7);
  double d, mx, my, mz, e;
  if (bulk) {
    const float* f = uf + o * kBulkF + cell;
    d = f[0];
    mx = f[8];
    my = f[16];
    mz = f[24];
    e = ud[o * kBulkD + cell];
  } else {
    const double* u = ud + o * 40 + cell;
    d = u[0];
    mx = u[8];
    my = u[16];
    mz = u[24];
    e = u[32];
  }
  const double vx = __ddiv_rn(mx, d), vy = __ddiv_rn(my, d), vz = __ddiv_rn(mz, d);
  const double v2 = __dadd_rn(__dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vy, vy)), __dmul_rn(vz, vz));
  const double ekin = __dmul_rn(__dmul_rn(0.5, d), v2);
  const double p = __dmul_rn(gm1, __dsub_rn(e, ekin));
  uint32_t* q = dst + o * 40 + cell;
  q[0] = __float_as_uint(__double2float_rn(d));
  q[8] = __float_as_uint(__double2float_rn(vx));
  q[16] = __float_as_uint(__double2float_rn(vy));
  q[24] = __float_as_uint(__double2float_rn(vz));
  q[32] = __float_as_uint(__double2float_rn(p));
}

// backup_hydro payload of an FP32-bulk state: uold(1:8, 1:5) per oct as
// float64 (rho and momenta widened exactly), written as 32-bit word pairs (a
// level starts 4-byte aligned in the file).  One thread per cell.
__global__ void state_image_kernel(const double* __restrict__ ue, const float* __restrict__ uf, long long noct,
                                   uint32_t* __restrict__ dst) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= noct * 8) return;
  const long long o = i >> 3;
  const int cell = (int)(i & 7);
  const float* f = uf + o * kBulkF + cell;
  double v[5];
#pragma unroll
  for (int k = 0; k < 4; ++k) v[k] = (double)f[8 * k];
  v[4] = ue[o * kBulkD + cell];
  uint32_t* w = dst + o * 80 + 2 * cell;
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v[k]);
    w[16 * k] = (uint32_t)b;
    w[16 * k + 1] = (uint32_t)(b >> 32);
  }
}

// Restart into an FP32-bulk state: the inverse of state_image_kernel, rho and
// momenta rounded to float32 as the mesh upload does.
__global__ void state_restore_kernel(const uint32_t* __restrict__ src, long long noct, float* __restrict__ uf,
                                     double* __restrict__ ue) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= noct * 8) return;
  const long long o = i >> 3;
  const int cell = (int)(i & 7);
  const uint32_t* w = src + o * 80 + 2 * cell;
  double v[5];
#pragma unroll
  for (int k = 0; k < 5; ++k)
    v[k] = __longlong_as_double((long long)((unsigned long long)w[16 * k] |
                                            ((unsigned long long)w[16 * k + 1] << 32)));
  float* f = uf + o * kBulkF + cell;
#pragma unroll
  for (int k = 0; k < 4; ++k) f[8 * k] = (float)v[k];
  ue[o * kBulkD + cell] = v[4];
}

bool valid_kind(int kind) {
  return kind == RH_FILE_AMR || kind == RH_FILE_HYDRO_BACKUP || kind == RH_FILE_HYDRO_OUTPUT;
}

long long header_bytes(int kind, int nlev) { return 4LL * ((kind == RH_FILE_AMR ? 3 : 4) + nlev); }

long long record_bytes(int kind) {
  return kind == RH_FILE_AMR ? 16 : (kind == RH_FILE_HYDRO_BACKUP ? 320 : 160);
}

unsigned blocks_for(long long n, int threads) { return (unsigned)((n + threads - 1) / threads); }

ImageSrc context_source() {
  Context& c = ctx();
  ImageSrc s;
  s.ud = c.ud[c.cur];
  s.uf = c.uf[c.cur];
  s.bulk = c.precision == RH_PREC_FP32_BULK;
  s.levelmin = c.levelmin;
  s.levelmax = c.levelmax;
  for (int l = c.levelmin; l <= c.levelmax; ++l) {
    s.oct0.push_back(c.noct[l] > 0 ? c.head[l] - 1 : 0);
    s.noct.push_back(c.noct[l]);
  }
  s.grid = c.grid.data();
  return s;
}

int check_mesh(const char* who) {
  Context& c = ctx();
  if (!c.inited || !c.have_mesh) {
    set_error("%s: rh_init and rh_set_mesh first", who);
    return RH_ESTATE;
  }
  return RH_OK;
}

}  // namespace

long long image_bytes(int kind, const ImageSrc& s) {
  long long n = 0;
  for (long long k : s.noct) n += k;
  return header_bytes(kind, (int)s.noct.size()) + record_bytes(kind) * n;
}

int build_image(int kind, const ImageSrc& s, double gamma, const void** dimage, long long* nbytes) {
  Context& c = ctx();
  if (!valid_kind(kind)) {
    set_error("file image: unknown kind %d", kind);
    return RH_EINVAL;
  }
  const int nlev = (int)s.noct.size();
  const long long hsize = header_bytes(kind, nlev), total = image_bytes(kind, s);
  for (long long k : s.noct)
    if (k > 2147483647LL) {
      set_error("file image: a level holds more than 2^31-1 octs (the header's int32 noct)");
      return RH_EINVAL;
    }
  int rc = ensure_image((size_t)total);
  if (rc) return rc;
  char* img = (char*)g_image;
  // header (ints as write(ilun) puts them in a stream file)
  std::vector<int32_t> hdr;
  hdr.push_back(3);
  if (kind != RH_FILE_AMR) hdr.push_back(5);
  hdr.push_back(s.levelmin);
  hdr.push_back(s.levelmax);
  for (long long k : s.noct) hdr.push_back((int32_t)k);
  if (kind == RH_FILE_AMR) {
    // per oct: ckey(1:3), refined bits (ibset(refined_int, ind-1))
    long long n = 0;
    for (long long k : s.noct) n += k;
    hdr.reserve(hdr.size() + 4 * (size_t)n);
    for (int li = 0; li < nlev; ++li) {
      for (long long i = 0; i < s.noct[li]; ++i) {
        if (s.grid) {
          const rh_oct& o = s.grid[s.oct0[li] + i];
          int32_t bits = 0;
          for (int ind = 0; ind < 8; ++ind)
            if (o.refined[ind]) bits |= 1 << ind;
          hdr.push_back(o.ckey[0]);
          hdr.push_back(o.ckey[1]);
          hdr.push_back(o.ckey[2]);
          hdr.push_back(bits);
        } else {  // one row-major box level
          const long long x = i % s.nxo, y = (i / s.nxo) % s.nyo, z = i / (s.nxo * s.nyo);
          hdr.push_back((int32_t)x);
          hdr.push_back((int32_t)y);
          hdr.push_back((int32_t)z);
          hdr.push_back(0);
        }
      }
    }
    RH_CUDA(cudaMemcpyAsync(img, hdr.data(), sizeof(int32_t) * hdr.size(), cudaMemcpyHostToDevice, c.stream));
  } else {
    RH_CUDA(cudaMemcpyAsync(img, hdr.data(), (size_t)hsize, cudaMemcpyHostToDevice, c.stream));
    long long off = hsize;
    const int threads = 256;
    for (int li = 0; li < nlev; ++li) {
      const long long n = s.noct[li], o0 = s.oct0[li];
      if (n == 0) continue;
      uint32_t* dst = (uint32_t*)(img + off);
      if (kind == RH_FILE_HYDRO_OUTPUT) {
        const double* ud = s.bulk ? s.ud + o0 * kBulkD : s.ud + o0 * 40;
        const float* uf = s.bulk ? s.uf + o0 * kBulkF : nullptr;
        prim_image_kernel<<<blocks_for(n * 8, threads), threads, 0, c.stream>>>(ud, uf, s.bulk, n, gamma - 1.0,
                                                                               dst);
      } else if (s.bulk) {
        state_image_kernel<<<blocks_for(n * 8, threads), threads, 0, c.stream>>>(s.ud + o0 * kBulkD,
                                                                               s.uf + o0 * kBulkF, n, dst);
      } else {
        RH_CUDA(cudaMemcpyAsync(dst, s.ud + o0 * 40, (size_t)n * 320, cudaMemcpyDeviceToDevice, c.stream));
      }
      RH_CUDA(cudaGetLastError());
      off += n * record_bytes(kind);
    }
  }
  RH_CUDA(cudaStreamSynchronize(c.stream));
  *dimage = g_image;
  *nbytes = total;
  return RH_OK;
}

int image_to_host(const void* dimage, long long nbytes, void* host_buf, long long cap) {
  Context& c = ctx();
  if (!host_buf || cap < nbytes) {
    set_error("file image: buffer of %lld bytes, the image needs %lld", cap, nbytes);
    return RH_EINVAL;
  }
  RH_CUDA(cudaMemcpyAsync(host_buf, dimage, (size_t)nbytes, cudaMemcpyDeviceToHost, c.stream));
  RH_CUDA(cudaStreamSynchronize(c.stream));
  return RH_OK;
}

void free_image_buffer() {
  cudaFree(g_image);
  g_image = nullptr;
  g_image_cap = 0;
}

}  // namespace rh

using namespace rh;

extern "C" {

int rh_file_size(int kind, long long* nbytes) {
  int rc = check_mesh("rh_file_size");
  if (rc) return rc;
  if (!nbytes || !valid_kind(kind)) {
    set_error("rh_file_size: bad kind %d or null output", kind);
    return RH_EINVAL;
  }
  *nbytes = image_bytes(kind, context_source());
  return RH_OK;
}

int rh_file_image_device(int kind, double gamma, const void** dimage, long long* nbytes) {
  int rc = check_mesh("rh_file_image_device");
  if (rc) return rc;
  if (!dimage || !nbytes) {
    set_error("rh_file_image_device: null output");
    return RH_EINVAL;
  }
  return build_image(kind, context_source(), gamma, dimage, nbytes);
}

int rh_file_image(int kind, double gamma, void* host_buf, long long cap, long long* nbytes) {
  int rc = check_mesh("rh_file_image");
  if (rc) return rc;
  if (!nbytes) {
    set_error("rh_file_image: null output");
    return RH_EINVAL;
  }
  const ImageSrc s = context_source();
  if (!valid_kind(kind)) {
    set_error("rh_file_image: unknown kind %d", kind);
    return RH_EINVAL;
  }
  const long long need = image_bytes(kind, s);
  *nbytes = need;
  if (!host_buf || cap < need) {
    set_error("rh_file_image: buffer of %lld bytes, the image needs %lld", cap, need);
    return RH_EINVAL;
  }
  const void* d = nullptr;
  long long n = 0;
  rc = build_image(kind, s, gamma, &d, &n);
  if (rc) return rc;
  return image_to_host(d, n, host_buf, cap);
}

int rh_restore_hydro(const void* image, long long nbytes) {
  int rc = check_mesh("rh_restore_hydro");
  if (rc) return rc;
  Context& c = ctx();
  if (!image || nbytes < 16) {
    set_error("rh_restore_hydro: no image");
    return RH_EINVAL;
  }
  int32_t h[4];
  std::memcpy(h, image, sizeof(h));
  if (h[0] != 3 || h[1] != 5 || h[2] != c.levelmin || h[3] != c.levelmax) {
    set_error("rh_restore_hydro: header (ndim %d, nvar %d, levels %d..%d) does not match the mesh (3, 5, %d..%d)",
              h[0], h[1], h[2], h[3], c.levelmin, c.levelmax);
    return RH_EINVAL;
  }
  const int nlev = c.levelmax - c.levelmin + 1;
  const long long hsize = header_bytes(RH_FILE_HYDRO_BACKUP, nlev);
  if (nbytes < hsize) {
    set_error("rh_restore_hydro: image shorter than its header");
    return RH_EINVAL;
  }
  std::vector<int32_t> noct((size_t)nlev);
  std::memcpy(noct.data(), (const char*)image + 16, sizeof(int32_t) * nlev);
  long long total = 0;
  for (int li = 0; li < nlev; ++li) {
    if (noct[li] != c.noct[c.levelmin + li]) {
      set_error("rh_restore_hydro: level %d has %d octs in the image, %d in the mesh", c.levelmin + li, noct[li],
                c.noct[c.levelmin + li]);
      return RH_EINVAL;
    }
    total += noct[li];
  }
  if (nbytes != hsize + 320 * total) {
    set_error("rh_restore_hydro: image of %lld bytes, header implies %lld", nbytes, hsize + 320 * total);
    return RH_EINVAL;
  }
  const char* payload = (const char*)image + hsize;
  if (c.precision == RH_PREC_FP64) {
    long long off = 0;
    for (int li = 0; li < nlev; ++li) {
      const long long n = noct[li], o0 = c.head[c.levelmin + li] - 1;
      if (n)
        RH_CUDA(cudaMemcpyAsync(c.ud[c.cur] + o0 * 40, payload + off, (size_t)n * 320, cudaMemcpyHostToDevice,
                                c.stream));
      off += n * 320;
    }
  } else {
    rc = ensure_image((size_t)(320 * total));
    if (rc) return rc;
    RH_CUDA(cudaMemcpyAsync(g_image, payload, (size_t)(320 * total), cudaMemcpyHostToDevice, c.stream));
    long long off = 0;
    const int threads = 256;
    for (int li = 0; li < nlev; ++li) {
      const long long n = noct[li], o0 = c.head[c.levelmin + li] - 1;
      if (n) {
        state_restore_kernel<<<blocks_for(n * 8, threads), threads, 0, c.stream>>>(
            (const uint32_t*)((const char*)g_image + off), n, c.uf[c.cur] + o0 * kBulkF, c.ud[c.cur] + o0 * kBulkD);
        RH_CUDA(cudaGetLastError());
      }
      off += n * 320;
    }
  }
  RH_CUDA(cudaStreamSynchronize(c.stream));
  std::fill(c.cfl_on_unew.begin(), c.cfl_on_unew.end(), 0);
  std::fill(c.cfl_on_uold.begin(), c.cfl_on_uold.end(), 0);
  return RH_OK;
}

}  // extern "C"
