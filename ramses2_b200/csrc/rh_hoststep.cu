// rh_hoststep.cu — one coarse step of a single-level mesh whose state lives in
// host memory, with the host-to-device copy, the Godunov pencils and the
// device-to-host copy overlapped (PCIe runs both directions at once).
//
// The level's octs are cut into chunks of consecutive octs (in the reference's
// oct order); chunks are uploaded in the z-major order of their centres on one
// copy stream.  A pencil can run once every oct of its neighbourhood (its
// table) has arrived: pencils are grouped by the upload position of the last
// chunk they need and each group is launched when that chunk is on the device
// (FP32-bulk: packed into its oct records).  A chunk is downloaded on a second
// copy stream once the last group that writes one of its octs has finished.
// Four streams in all (library, upload, unpack, download): spreading the
// groups over eight more streams, beyond CUDA's default eight hardware work
// queues, made the copies queue behind kernels (26.6 ms per 256^3 step
// against 18.1).
// The pencil kernel is the one rh_coarse_step runs (the level's tile shape),
// launched group by group over the schedule's own pencil tables, 2 (FP32-bulk)
// or 8 (FP64) layers deep.  A cell's update does not depend on where pencils
// start and end, so the new state is bitwise that of rh_set_grid_device +
// rh_coarse_step + rh_transfer_grid_host, and so is the next dt (a minimum);
// the conserved totals of the fused CFL epilogue are summed over other
// pencils, so they agree to rounding.
//
// The step's dt must be known before the first pencil runs.  A host that
// loops passes the dt_next of its previous call: min(dx/smallc, courant dt)
// of the state that call returned, computed on the device by the step's
// fused CFL epilogue (the reference's newdt_fine takes the courant_fine of
// the same state at the start of the next step).  Without it (dt <= 0) the
// CFL reduction of the uploaded state runs after the whole upload, and only
// the download overlaps the pencils.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "ramses_hydro_ext.h"
#include "rh_internal.h"

namespace rh {

struct HostStepSched {
  // what the schedule was built for: level, kernel tile shape, precision
  int level = -1, txo = 0, tyo = 0, minb = 0, precision = -1;
  long long noct = 0;
  // the schedule's own pencil tables: the level's tile shape, sched_lz() layers deep
  LevelTables T;
  int npencil = 0;
  // chunks: [k*C, min((k+1)*C, noct)) octs; uploaded in the order up_order
  long long C = 0;
  int nchunk = 0;
  std::vector<int> up_order;   // upload position -> chunk
  std::vector<int> gstart;     // [nchunk+1]: group r = pencils [gstart[r], gstart[r+1]) of the group order
  std::vector<int> down_order; // chunks in download order
  std::vector<int> fin;        // [chunk]: upload position after whose group the chunk is final
  int4* d_phdr = nullptr;      // pencil headers / table offsets in group order
  long long* d_poff = nullptr;
  double* d_partial = nullptr; // fused CFL partials in group order
  cudaStream_t up = nullptr, down = nullptr, unpk = nullptr;
  std::vector<cudaEvent_t> ev_up, ev_grp, ev_unpk;
  cudaEvent_t ev_start = nullptr, ev_down = nullptr;
};

namespace {

// Pencils this deep: a pencil needs its neighbourhood and a chunk waits for
// the pencils that write it, so shallow pencils start earlier and release
// chunks sooner; the pencils' extra halo work is hidden behind the copies.
// FP32-bulk takes 2 layers, FP64 8: on a 256^3 step 2 layers brought the
// FP32-bulk step from 18.7 to 18.2 ms (the first chunks go back sooner, and
// the extra halo work of its fast kernel stays hidden behind the copies) and
// the FP64 one from 16.3 to 18.2 ms (its kernel, twice as slow, no longer
// keeps pace).
int sched_lz(int precision) { return precision == RH_PREC_FP32_BULK ? 2 : 8; }
// 128 chunks of 16,384 octs (5.2 MB of FP64 state per copy) for a 256^3
// level: on one box 18.8-18.9 ms per FP32-bulk step, against 18.3-19.6 with
// 256 chunks and 20-21 with 64 (fewer chunks leave a longer tail of downloads
// after the last upload; more add per-copy cost on a link already carrying
// both directions).
constexpr long long kChunkOcts = 16384;
constexpr int kMaxChunks = 128;

HostStepSched*& sched_ptr() {
  static HostStepSched* s = nullptr;
  return s;
}

void free_sched(HostStepSched* s) {
  if (!s) return;
  cudaFree(s->T.d_ptab);
  cudaFree(s->d_phdr);
  cudaFree(s->d_poff);
  cudaFree(s->d_partial);
  for (auto* v : {&s->ev_up, &s->ev_grp, &s->ev_unpk})
    for (cudaEvent_t e : *v) cudaEventDestroy(e);
  if (s->ev_start) cudaEventDestroy(s->ev_start);
  if (s->ev_down) cudaEventDestroy(s->ev_down);
  for (cudaStream_t st : {s->up, s->down, s->unpk})
    if (st) cudaStreamDestroy(st);
  delete s;
}

int build_sched(int l, HostStepSched& S) {
  Context& c = ctx();
  const long long N = c.noct[l];
  const long long o0 = c.head[l] - 1;  // 0 for the single level of a mesh
  const TileCfg& main = c.cfg;
  TileCfg cfg = main;
  cfg.lz = sched_lz(c.precision);
  S.level = l;
  S.txo = main.txo;
  S.tyo = main.tyo;
  S.minb = main.minb;
  S.precision = c.precision;
  S.noct = N;
  S.T.cfg = cfg;
  int rc = build_complete_tables_device(l, cfg, S.T);
  if (rc) return rc;
  LevelTables& T = S.T;
  S.npencil = (int)T.phdr.size();
  S.nchunk = (int)std::max(1ll, std::min<long long>(kMaxChunks, (N + kChunkOcts - 1) / kChunkOcts));
  S.C = (N + S.nchunk - 1) / S.nchunk;
  S.nchunk = (int)((N + S.C - 1) / S.C);
  const int K = S.nchunk;
  // upload order: chunks by the z, y, x of their oct centres
  std::vector<double> cen(3 * (size_t)K, 0.0);
  std::vector<long long> cnt(K, 0);
  for (long long o = 0; o < N; ++o) {
    const int k = (int)(o / S.C);
    for (int d = 0; d < 3; ++d) cen[3 * k + d] += c.grid[o0 + o].ckey[d];
    cnt[k]++;
  }
  S.up_order.resize(K);
  std::iota(S.up_order.begin(), S.up_order.end(), 0);
  std::stable_sort(S.up_order.begin(), S.up_order.end(), [&](int a, int b) {
    for (int d = 2; d >= 0; --d) {
      const double x = cen[3 * a + d] / cnt[a], y = cen[3 * b + d] / cnt[b];
      if (x != y) return x < y;
    }
    return false;
  });
  std::vector<int> pos(K);
  for (int r = 0; r < K; ++r) pos[S.up_order[r]] = r;
  // every pencil's neighbourhood from its oct table
  std::vector<int> tab(T.ntab);
  RH_CUDA(cudaMemcpy(tab.data(), T.d_ptab, sizeof(int) * T.ntab, cudaMemcpyDeviceToHost));
  const int OW = cfg.txo + 2, NSLOT = (cfg.txo + 2) * (cfg.tyo + 2);
  std::vector<int> need(S.npencil, 0);
  S.fin.assign(K, -1);
  for (int p = 0; p < S.npencil; ++p) {
    const int4 h = T.phdr[p];
    const int* t = tab.data() + T.poff[p];
    const long long nent = (long long)(h.w + 2) * NSLOT;
    int nd = 0;
    for (long long e = 0; e < nent; ++e)
      if (t[e] >= 0) nd = std::max(nd, pos[(int)((t[e] - o0) / S.C)]);
    need[p] = nd;
    // the octs this pencil writes: interior rows and columns inside the level
    for (int r = 1; r <= h.w; ++r)
      for (int iy = 0; iy < cfg.tyo; ++iy)
        for (int ix = 0; ix < cfg.txo; ++ix) {
          if (h.x + ix >= T.nxo || h.y + iy >= T.nyo) continue;
          const int e = t[(long long)r * NSLOT + (ix + 1) + OW * (iy + 1)];
          if (e < 0) continue;
          const int k = (int)((e - o0) / S.C);
          S.fin[k] = std::max(S.fin[k], nd);
        }
  }
  for (int k = 0; k < K; ++k)
    if (S.fin[k] < 0) S.fin[k] = K - 1;  // written by no pencil: download last
  std::vector<int> porder(S.npencil);
  std::iota(porder.begin(), porder.end(), 0);
  std::stable_sort(porder.begin(), porder.end(), [&](int a, int b) { return need[a] < need[b]; });
  S.gstart.assign(K + 1, 0);
  for (int p = 0; p < S.npencil; ++p) S.gstart[need[p] + 1]++;
  for (int g = 0; g < K; ++g) S.gstart[g + 1] += S.gstart[g];
  S.down_order.resize(K);
  std::iota(S.down_order.begin(), S.down_order.end(), 0);
  std::stable_sort(S.down_order.begin(), S.down_order.end(), [&](int a, int b) {
    return S.fin[a] != S.fin[b] ? S.fin[a] < S.fin[b] : pos[a] < pos[b];
  });
  std::vector<int4> ph(S.npencil);
  std::vector<long long> po(S.npencil);
  for (int i = 0; i < S.npencil; ++i) {
    ph[i] = T.phdr[porder[i]];
    po[i] = T.poff[porder[i]];
  }
  RH_CUDA(cudaMalloc(&S.d_phdr, sizeof(int4) * std::max(1, S.npencil)));
  RH_CUDA(cudaMalloc(&S.d_poff, sizeof(long long) * std::max(1, S.npencil)));
  RH_CUDA(cudaMalloc(&S.d_partial, sizeof(double) * 5 * std::max(1, S.npencil)));
  RH_CUDA(cudaMemcpy(S.d_phdr, ph.data(), sizeof(int4) * S.npencil, cudaMemcpyHostToDevice));
  RH_CUDA(cudaMemcpy(S.d_poff, po.data(), sizeof(long long) * S.npencil, cudaMemcpyHostToDevice));
  RH_CUDA(cudaStreamCreateWithFlags(&S.up, cudaStreamNonBlocking));
  RH_CUDA(cudaStreamCreateWithFlags(&S.down, cudaStreamNonBlocking));
  RH_CUDA(cudaStreamCreateWithFlags(&S.unpk, cudaStreamNonBlocking));
  for (auto* v : {&S.ev_up, &S.ev_grp, &S.ev_unpk}) {
    v->assign(K, nullptr);
    for (int k = 0; k < K; ++k) RH_CUDA(cudaEventCreateWithFlags(&(*v)[k], cudaEventDisableTiming));
  }
  RH_CUDA(cudaEventCreateWithFlags(&S.ev_start, cudaEventDisableTiming));
  RH_CUDA(cudaEventCreateWithFlags(&S.ev_down, cudaEventDisableTiming));
  return RH_OK;
}

}  // namespace

void free_host_schedule() {
  free_sched(sched_ptr());
  sched_ptr() = nullptr;
}

}  // namespace rh

using namespace rh;

extern "C" {

int rh_coarse_step_host(const rh_hydro_params* p, const double* host_in, double* host_out, double* dt,
                        double* dt_next) {
  Context& c = ctx();
  if (!c.inited || !c.have_mesh) {
    set_error("rh_coarse_step_host: no mesh (rh_init / rh_set_mesh first)");
    return RH_ESTATE;
  }
  if (!p || !host_in || !host_out || !dt) {
    set_error("rh_coarse_step_host: null argument");
    return RH_EINVAL;
  }
  int nlev = 0, l = -1;
  for (int k = c.levelmin; k <= c.levelmax; ++k)
    if (c.noct[k] > 0) {
      nlev++;
      l = k;
    }
  const double dx = l >= 0 ? c.boxlen / std::ldexp(1.0, l) : 0.0;
  const double g[3] = {c.gravity[0], c.gravity[1], c.gravity[2]};
  int rc;
  if (nlev != 1 || c.noct[l] != c.ngridmax || c.nsubgrid != 1 || p->difmag > 0.0) {
    // several levels (or spare octs), or artificial diffusion: the same
    // calls one after the other
    if ((rc = rh_set_grid_device(host_in, c.ngridmax, 5, 8))) return rc;
    if ((rc = rh_coarse_step(p, dt, nullptr))) return rc;
    if ((rc = rh_transfer_grid_host(host_out, c.ngridmax, 5, 8))) return rc;
    if (dt_next) {
      double best = 1e300;
      for (int k = c.levelmin; k <= c.levelmax; ++k) {
        if (!c.noct[k]) continue;
        double m, ek, ei, em, d;
        const double dxk = c.boxlen / std::ldexp(1.0, k);
        if ((rc = rh_cmpdt(c.head[k], c.noct[k], dxk, p->gamma, p->smallr, p->smallc, p->courant_factor, g, &m,
                           &ek, &ei, &em, &d)))
          return rc;
        best = std::min(best, d);
      }
      *dt_next = best;
    }
    return RH_OK;
  }
  HostStepSched*& sp = sched_ptr();
  {
    if (sp && (sp->level != l || sp->txo != c.cfg.txo || sp->tyo != c.cfg.tyo || sp->minb != c.cfg.minb ||
               sp->precision != c.precision || sp->noct != c.noct[l]))
      free_host_schedule();
    if (!sp) {
      sp = new HostStepSched();
      if ((rc = build_sched(l, *sp))) {
        free_host_schedule();
        return rc;
      }
    }
  }
  HostStepSched& S = *sp;
  const bool bulk = c.precision == RH_PREC_FP32_BULK;
  const long long N = c.noct[l];
  double* stage = nullptr;
  if (bulk && (rc = stage64(N, &stage))) return rc;
  const int K = S.nchunk;
  auto chunk_octs = [&](int k) { return std::min(S.C, N - k * S.C); };
  // everything queued before this call is done with the state buffers first
  RH_CUDA(cudaEventRecord(S.ev_start, c.stream));
  for (cudaStream_t st : {S.up, S.down, S.unpk}) RH_CUDA(cudaStreamWaitEvent(st, S.ev_start, 0));
  const int cur = c.cur, nxt = 1 - c.cur;
  for (int r = 0; r < K; ++r) {
    const int k = S.up_order[r];
    const long long o = k * S.C, n = chunk_octs(k);
    double* dst = bulk ? stage + o * 40 : c.ud[cur] + o * 40;
    RH_CUDA(cudaMemcpyAsync(dst, host_in + o * 40, sizeof(double) * 40 * n, cudaMemcpyHostToDevice, S.up));
    RH_CUDA(cudaEventRecord(S.ev_up[r], S.up));
  }
  // chunk ready for the pencils (FP32-bulk: packed into oct records), in
  // upload order on the library stream
  auto ready = [&](int r) -> int {
    RH_CUDA(cudaStreamWaitEvent(c.stream, S.ev_up[r], 0));
    if (bulk) {
      const int k = S.up_order[r];
      const long long o = k * S.C, n = chunk_octs(k);
      pack_bulk_kernel<<<(unsigned)((n * 8 + 255) / 256), 256, 0, c.stream>>>(
          stage + o * 40, c.uf[cur] + o * kBulkF, c.ud[cur] + o * kBulkD, n);
      RH_CUDA(cudaGetLastError());
    }
    return RH_OK;
  };
  // courant_fine keys of the fused CFL epilogue (as rh_cmpdt records them)
  const double key[8] = {dx, p->gamma, p->smallr, p->smallc, p->courant_factor, g[0], g[1], g[2]};
  std::copy(key, key + 8, &c.cfl_keys[8 * l]);
  double step_dt = *dt;
  const bool given = step_dt > 0;
  if (!given) {
    // no dt from the host: the CFL of the uploaded state after the whole upload
    for (int r = 0; r < K; ++r)
      if ((rc = ready(r))) return rc;
    c.cfl_on_uold[l] = 0;
    c.cfl_on_unew[l] = 0;
    double m, ek, ei, em;
    if ((rc = rh_cmpdt(c.head[l], (int)N, dx, p->gamma, p->smallr, p->smallc, p->courant_factor, g, &m, &ek, &ei,
                       &em, &step_dt)))
      return rc;
  }
  const double smax_cap = p->courant_factor * dx / step_dt;
  for (int r = 0; r < K; ++r) {
    if (given && (rc = ready(r))) return rc;
    const int n = S.gstart[r + 1] - S.gstart[r];
    if (n > 0) {
      PencilRange R{S.d_phdr + S.gstart[r], S.d_poff + S.gstart[r], S.T.d_ptab, S.d_partial + 5ll * S.gstart[r], n,
                    nullptr};
      if ((rc = launch_level(l, p->gamma, p->smallr, p->smallc, step_dt, dx, smax_cap, p->slope_type, p->riemann, g,
                             true, false, &R)))
        return rc;
    }
    RH_CUDA(cudaEventRecord(S.ev_grp[r], c.stream));
  }
  // the fused CFL values of the new state (fixed reduction order of the schedule's pencils)
  const double cdx_smallc = p->courant_factor * dx / p->smallc;
  reduce_partials_kernel<<<1, 1024, 0, c.stream>>>(S.d_partial, S.npencil, cdx_smallc, c.d_cfl + 5 * l);
  c.cfl_gen++;
  RH_CUDA(cudaGetLastError());
  // downloads of the finished chunks: FP32-bulk records unpacked to FP64 on
  // their own stream, so the copy stream only copies
  for (int i = 0; i < K; ++i) {
    const int k = S.down_order[i];
    const long long o = k * S.C, n = chunk_octs(k);
    const double* src = c.ud[nxt] + o * 40;
    if (bulk) {
      RH_CUDA(cudaStreamWaitEvent(S.unpk, S.ev_grp[S.fin[k]], 0));
      unpack_bulk_kernel<<<(unsigned)((n * 8 + 255) / 256), 256, 0, S.unpk>>>(stage + o * 40, c.uf[nxt] + o * kBulkF,
                                                                            c.ud[nxt] + o * kBulkD, n);
      RH_CUDA(cudaGetLastError());
      RH_CUDA(cudaEventRecord(S.ev_unpk[i], S.unpk));
      RH_CUDA(cudaStreamWaitEvent(S.down, S.ev_unpk[i], 0));
      src = stage + o * 40;
    } else {
      RH_CUDA(cudaStreamWaitEvent(S.down, S.ev_grp[S.fin[k]], 0));
    }
    RH_CUDA(cudaMemcpyAsync(host_out + o * 40, src, sizeof(double) * 40 * n, cudaMemcpyDeviceToHost, S.down));
  }
  RH_CUDA(cudaEventRecord(S.ev_down, S.down));
  RH_CUDA(cudaStreamWaitEvent(c.stream, S.ev_down, 0));
  double h[5];
  RH_CUDA(cudaMemcpyAsync(h, c.d_cfl + 5 * l, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
  RH_CUDA(cudaStreamSynchronize(c.stream));
  // the new state is current (set_uold as a buffer swap); its CFL values are cached
  c.cur = nxt;
  c.unew_pending[l] = 0;
  c.unew_written[l] = 0;
  c.unew_copied[l] = 0;
  c.cfl_on_uold[l] = 1;
  c.cfl_on_unew[l] = 0;
  *dt = step_dt;
  if (dt_next) *dt_next = std::min(dx / p->smallc, h[4]);
  int err = 0;
  RH_CUDA(cudaMemcpy(&err, c.d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) {
    cudaMemset(c.d_err, 0, sizeof(int));
    set_error("device wait bound exceeded in a pencil kernel (error word %d)", err);
    return RH_ETIMEDOUT;
  }
  return RH_OK;
}

}  // extern "C"
