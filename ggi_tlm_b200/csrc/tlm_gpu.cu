// tlm_gpu.cu -- C-ABI (include/tlm_gpu.h) over the sm_100a SCN-TLM kernels.
//
// A handle owns one mesh: the ping-pong reflected-pulse planes, the compact
// special-cell tables (per-32-cell bit masks + prefix counts + one int4
// record per special cell), the PML and Z-filter state, the per-step cell
// excitation table, the cell-output ring and the DFT accumulators.  Tables
// are assembled on the host from the reference's module arrays at the first
// run (or explicit finalisation) and uploaded once.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/tlm_gpu.h"
#include "tlm_kernels.cuh"

namespace {

thread_local std::string g_last_error;

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

#define CK(call)                                                                                  \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess) return fail(TLM_E_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                                       __FILE__, __LINE__);                                       \
  } while (0)

// ---------------------------------------------------------------------------
// Device-memory cache.  Buffers released by destroyed meshes and by rebuilt
// batch lists are kept per device and handed out again to later allocations
// of a similar size, so a serving loop that creates and destroys meshes all
// the time stops paying for cudaMalloc/cudaFree (a single cudaFree of a
// large buffer took up to 0.6 s on B200).  Blocks of destroyed meshes and
// batches are released after their streams were synchronised and can be
// reused at once.  A buffer replaced while work may still be in flight (a
// batch's lists rebuilt between graph launches) may still be read, so the
// first reuse after such a release synchronises the device first, as
// cudaFree would have.  The cache holds
// at most TLM_POOL_CACHE_BYTES (default 16 GiB) per device; beyond that, and
// on tlm_gpu_pool_release, blocks go back to the driver.
// ---------------------------------------------------------------------------
namespace pool {
std::mutex mu;
std::map<int, std::multimap<size_t, void *>> blocks;  // device -> (capacity, pointer)
std::map<int, size_t> cached;                         // device -> cached bytes
std::map<int, bool> released_since_sync;              // device -> a release happened since the last sync

size_t cache_limit() {
  static size_t lim = [] {
    const char *e = getenv("TLM_POOL_CACHE_BYTES");
    return e ? (size_t)strtoull(e, nullptr, 10) : ((size_t)16 << 30);
  }();
  return lim;
}

size_t round_up(size_t b) {
  const size_t g = b <= ((size_t)1 << 20) ? 4096 : ((size_t)2 << 20);
  return (b + g - 1) / g * g;
}

// A block of at least `bytes` on the current device; its capacity in *cap.
cudaError_t alloc(size_t bytes, void **p, size_t *cap) {
  int dev = 0;
  cudaGetDevice(&dev);
  const size_t want = round_up(bytes);
  {
    std::lock_guard<std::mutex> lk(mu);
    auto &bl = blocks[dev];
    auto it = bl.lower_bound(want);
    if (it != bl.end() && it->first <= want + want / 4) {
      if (released_since_sync[dev]) {
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) return e;
        released_since_sync[dev] = false;
      }
      *p = it->second;
      *cap = it->first;
      cached[dev] -= it->first;
      bl.erase(it);
      return cudaSuccess;
    }
  }
  cudaError_t e = cudaMalloc(p, want);
  if (e == cudaErrorMemoryAllocation) {  // give the cache back to the driver and retry
    cudaGetLastError();
    std::lock_guard<std::mutex> lk(mu);
    for (auto &kv : blocks[dev]) cudaFree(kv.second);
    blocks[dev].clear();
    cached[dev] = 0;
    e = cudaMalloc(p, want);
  }
  *cap = want;
  return e;
}

// idle: no kernel can still use the block (its streams were synchronised)
void release(int dev, void *p, size_t cap, bool idle) {
  if (!p) return;
  std::lock_guard<std::mutex> lk(mu);
  if (cached[dev] + cap > cache_limit()) {
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != dev) cudaSetDevice(dev);
    cudaFree(p);
    if (cur != dev) cudaSetDevice(cur);
    return;
  }
  blocks[dev].emplace(cap, p);
  cached[dev] += cap;
  if (!idle) released_since_sync[dev] = true;
}

void release_all() {
  std::lock_guard<std::mutex> lk(mu);
  int cur = 0;
  cudaGetDevice(&cur);
  for (auto &dv : blocks) {
    cudaSetDevice(dv.first);
    for (auto &kv : dv.second) cudaFree(kv.second);
    dv.second.clear();
    cached[dv.first] = 0;
  }
  cudaSetDevice(cur);
}

size_t cached_bytes() {
  std::lock_guard<std::mutex> lk(mu);
  size_t t = 0;
  for (auto &kv : cached) t += kv.second;
  return t;
}
}  // namespace pool

struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;  // requested
  size_t cap = 0;    // capacity of the cached block
  int dev = 0;
  // owners synchronise their streams before they are destroyed
  ~DevBuf() { pool::release(dev, p, cap, true); }
};

// Allocate `bytes` into b from the device cache (the current device).
cudaError_t buf_alloc(DevBuf &b, size_t bytes) {
  if (b.p) {
    pool::release(b.dev, b.p, b.cap, false);  // may still be read by work in flight
    b.p = nullptr;
  }
  b.bytes = bytes;
  cudaGetDevice(&b.dev);
  cudaError_t e = pool::alloc(bytes, &b.p, &b.cap);
  if (e != cudaSuccess) b.p = nullptr;
  return e;
}

// A second stream for the cell kernels that run beside the bulk kernel in a
// step.  The bulk, PML, PML-material and special-cell kernels all read the
// step-t links and write disjoint cells of step t+1, so the side kernels
// take the SM slots the persistent bulk kernel leaves free and its SMs as
// its CTAs retire, instead of waiting for its last wave.  The face kernel,
// which reads what all of them wrote, runs after the join.
struct SideStream {
  cudaStream_t s = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  int init() {
    if (s) return TLM_OK;
    CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
    return TLM_OK;
  }
  int begin(cudaStream_t main) {
    CK(cudaEventRecord(fork, main));
    CK(cudaStreamWaitEvent(s, fork, 0));
    return TLM_OK;
  }
  int end(cudaStream_t main) {
    CK(cudaEventRecord(join, s));
    CK(cudaStreamWaitEvent(main, join, 0));
    return TLM_OK;
  }
  ~SideStream() {
    if (fork) cudaEventDestroy(fork);
    if (join) cudaEventDestroy(join);
    if (s) cudaStreamDestroy(s);
  }
};

// Whether a mesh of n_cells runs its side kernels on the side stream.
// Measured on B200: it pays where the bulk kernel has few tiles per CTA
// (96^3 PML box -8 % per step, batches of serving meshes -1.4 %) and costs
// on large meshes, where the side kernels slow the bulk kernel down
// (256^3 +3 %, 512^3 +2 %).  TLM_SIDE_STREAM=0 / 1 forces it off / on.
bool side_stream_enabled(long long n_cells, bool batch) {
  const char *e = getenv("TLM_SIDE_STREAM");
  if (e && e[0] == '0') return false;
  if (e && e[0] == '1') return true;
  return batch || n_cells <= 4LL * 1024 * 1024;
}

struct Mesh {
  tlm_gpu_mesh_desc desc{};
  int Px = 0, Py = 0, Pz = 0;
  long long plane = 0;
  bool fp64 = false;
  bool finalized = false;
  int next_step = 1;  // next timestep to run (1-based)
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  bool timing = false;
  float last_total_ms = 0.f, last_cell_ms = 0.f;
  int timed_steps = 0;
  long long last_launches = 0;
  size_t dev_bytes = 0;

  // host copies of the reference arrays
  std::vector<int32_t> cell_code, sp_material, sp_pml, sp_exc, sp_out;
  int n_special = 0;
  bool have_cells = false;
  std::vector<tlm::MatDev> mats;
  std::vector<double> pml_params;
  std::vector<double> pml_sigma;  // [n_pml_params][3] sx, sy, sz (PML cells in a material)
  int n_pml_params = 0;
  std::vector<int32_t> pml_cell_param;
  int n_pml_cells = 0;
  int n_fn = 0, n_fn_steps = 0;
  std::vector<double> fn_value, fn_value_face;
  std::vector<int32_t> pt_cell, pt_comp, pt_fn, pt_type;
  int n_exc_cells = 0;
  std::vector<int32_t> f_cx, f_cy, f_cz, f_dir, f_exc, f_out;
  std::vector<int32_t> f_mat;  // surface material per special face (empty: none)
  std::vector<int32_t> f_smat;  // signed thin-layer material per special face (empty: none)
  int wrap = 0;                 // wrapping boundaries: bit 0 x, bit 1 y, bit 2 z
  std::vector<tlm::ThinLayerDev> thin;  // thin-layer materials
  // point sources on faces (excitation face number, component 1..12, function, type)
  std::vector<int32_t> fpt_face, fpt_comp, fpt_fn, fpt_type;
  std::vector<int32_t> fpt_side;  // per face source: 0 both sides, 1 or 2 that side alone; empty: all 0
  std::vector<double> fpt_scale;  // per face source: factor on the function's value; empty: all 1
  // output points on faces (output face number, side 1/2, component 1..6)
  std::vector<int32_t> fpr_face, fpr_side, fpr_comp;
  int n_exc_faces = 0, n_out_faces = 0;
  int hs_n = 0;
  std::vector<int32_t> hs_face_exc, hs_norm;
  std::vector<double> hs_offset;
  double hs_Ei[3] = {0, 0, 0}, hs_Hi[3] = {0, 0, 0}, hs_offset_min = 0, hs_c = 0;
  int hs_fn = 0;
  bool hs_outer = false;             // the Huygens surface is the outer boundary
  std::vector<int32_t> hs_cell;      // outer: 4 per patch (cx, cy, cz 1-based, face code)
  int n_out_cells = 0;
  std::vector<int32_t> out_keep;     // per output cell: 1 keeps a time series (empty: all do)
  int n_hist = 0;                    // outputs that keep a time series
  std::vector<double> vdft_freq;     // frequency output volumes, one per frequency
  std::vector<int32_t> vdft_gate;    // 4 per volume: first, last, interval, component
  std::vector<int32_t> vdft_ptr, vdft_out;
  int vdft_entries = 0;
  std::vector<int32_t> osurf_gate;   // time-domain output surfaces: 5 per surface (first, last, interval,
                                     // component, both sides)
  std::vector<int32_t> osurf_ptr, osurf_fout, osurf_fcode;
  int osurf_entries = 0;
  size_t osurf_hist_len = 0;
  std::vector<int32_t> ovol_gate;     // time-domain output volumes: 5 per volume (first, last, interval,
                                     // component, kind)
  std::vector<int32_t> ovol_ptr, ovol_out;
  size_t ovol_hist_len = 0;
  std::vector<double> ps_freq;       // frequency-domain power surfaces, one per surface and frequency
  std::vector<int32_t> ps_ptr, ps_fout, ps_fcode;
  int ps_entries = 0;
  std::vector<int32_t> mode_comp, mode_ptr, mode_fout, mode_fcode;  // mode outputs
  std::vector<double> mode_w;
  std::vector<double> sar_freq;      // SAR volumes, one per frequency
  std::vector<int32_t> sar_ptr, sar_out;
  int sar_entries = 0;
  bool rcs_on = false;               // the RCS surface (rcs_surface)
  double rcs_theta = 0, rcs_phi = 0;
  int rcs_npc = 2, rcs_points = 0, rcs_offset = 0;
  std::vector<int32_t> rcs_fout, rcs_fcode;
  std::vector<double> rcs_dist;
  int n_dft = 0;
  std::vector<double> dft_freq;
  std::vector<int32_t> dft_comp, dft_ptr, dft_fout, dft_fcode;
  std::vector<int32_t> dft_gate;  // [n_dft][3] first, last, interval (empty: every step)

  // device buffers
  DevBuf links, seg_mask, seg_base, sp_rec, sp_pos, pml_state, pml_par, pml_ixt, filt, mats_d, exc_field, exc_type,
      cell_out, faces, face_io, face_hs, value_face, face_field, dft_entry, dft_phasor, dft_acc, d_base,
      pmm_pos, pmm_parmat, pmm_state, pmm_sigma, face_src, fpt_field_d, fpt_type_d, fprobe, fprobe_rec,
      ohs_face, ohs_offset, ff_entry, ff_phasor, ff_acc, cell_cur, out_hist, vdft_entry, vdft_gate_d, vdft_phasor,
      vdft_acc, osurf_entry, osurf_pos, osurf_dev, osurf_hist, rcs_face, rcs_dist_d, rcs_tc0, rcs_acc, ovol_dev,
      face_mat_d, face_smat_d, pml_cls_par, thin_d, thin_taps, ovol_cells, ovol_hist, sar_entry, sar_phasor, sar_acc, ps_entry, ps_phasor, ps_acc, mode_d, mode_face, mode_wd,
      mode_hist;
  int n_pt_rows = 0;
  int n_pmm = 0;  // PML cells inside a volume material
  int n_filt = 0, filt_eo = 0, filt_mo = 0;
  int dft_entries = 0;
  std::vector<double> ff_freq;                       // far-field surfaces, one per frequency
  std::vector<int32_t> ff_ptr, ff_fout, ff_fcode;
  int ff_entries = 0;
  int n_sp_dev = 0;  // non-PML special cells on the device list
  int n_pml_list = 0, n_pml_out = 0;
  tlm::PmlShell pml_shell{};  // .on when the PML cells form a box shell
  DevBuf pml_pos, pml_par16, pml_outmap;
  // bulk-kernel variant: 0 = register-pipelined kernel, 1..kNumVariants-1 = TMA-staged configurations
  int variant = 1;
  int n_sms = 148;
  std::vector<uint32_t> host_mask;  // per-32-element special-cell masks (for tile lists)
  DevBuf tiles, d_err;
  std::vector<int4> host_tiles;
  cudaStream_t batch_stream = nullptr;  // set while the mesh belongs to a batch
  int tiles_tile = 0;  // TILE the current list was built for
  int n_tiles = 0;
  bool dry_launch = false;
  int small_every = 0;       // set_small_to_zero: period in steps (0 = off)
  double small_value = 0.0;
  int pml_prefetch = 1200;  // blocks ahead for the PML state L2 prefetch (0 = off)
  bool pml_by_class = false;  // PML parameters loaded by distance class (pml_cls_par)
  uint32_t tx_pad = 0;        // tlm_gpu_set_test_wait_pad
  SideStream side;          // PML / PML-material / special kernels beside the bulk kernel
  bool side_on = false;

  // graph of kGraphSteps steps
  static constexpr int kGraphSteps = 8;
  cudaGraphExec_t graph = nullptr;
  long long graph_launches = 0;  // kernel launches in one replay of the graph
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<cudaEvent_t> kev;

  ~Mesh() {
    if (graph) cudaGraphExecDestroy(graph);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    for (auto e : kev) cudaEventDestroy(e);
    if (own_stream && stream) cudaStreamDestroy(stream);
  }
};

std::mutex g_mu;
std::map<int64_t, std::unique_ptr<Mesh>> g_meshes;
int64_t g_next = 1;

Mesh *get(int64_t h) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_meshes.find(h);
  return it == g_meshes.end() ? nullptr : it->second.get();
}

int dalloc(Mesh *m, DevBuf &b, size_t bytes) {
  if (b.p) m->dev_bytes -= b.bytes;
  cudaError_t e = buf_alloc(b, std::max<size_t>(bytes, 16));
  if (e != cudaSuccess) return fail(TLM_E_OOM, "device allocation of %zu bytes failed: %s", b.bytes, cudaGetErrorString(e));
  m->dev_bytes += b.bytes;
  return TLM_OK;
}

template <typename V>
int upload(Mesh *m, DevBuf &b, const std::vector<V> &v) {
  int rc = dalloc(m, b, v.size() * sizeof(V));
  if (rc) return rc;
  if (!v.empty()) CK(cudaMemcpy(b.p, v.data(), v.size() * sizeof(V), cudaMemcpyHostToDevice));
  return TLM_OK;
}

template <typename T>
tlm::MeshDev<T> mesh_dev(Mesh *m) {
  tlm::MeshDev<T> d{};
  d.nx = m->desc.nx;
  d.ny = m->desc.ny;
  d.nz = m->desc.nz;
  d.Px = m->Px;
  d.Py = m->Py;
  d.PxPy = (long long)m->Px * m->Py;
  d.plane = m->plane;
  const int VEC = sizeof(T) == 4 ? 4 : 2;
  d.chunks_per_plane = (m->desc.ny * m->Px) / VEC;
  d.segs_per_plane = (m->desc.ny * m->Px + 31) / 32;
  T *base = (T *)m->links.p;
  d.links0 = base;
  d.links1 = base + 12 * m->plane;
  for (int i = 0; i < 6; i++) d.R[i] = T(m->desc.R[i]);
  d.seg_mask = (const uint32_t *)m->seg_mask.p;
  d.seg_base = (const uint32_t *)m->seg_base.p;
  d.sp_rec = (const int4 *)m->sp_rec.p;
  d.sp_pos = (const int4 *)m->sp_pos.p;
  d.pml_state = (typename tlm::PmlTypes<T>::state *)m->pml_state.p;
  d.n_pml = m->n_pml_cells;
  d.pml_par = (const double *)m->pml_par.p;
  d.pml_ixt = (typename tlm::PmlTypes<T>::state *)m->pml_ixt.p;
  d.filt = (double *)m->filt.p;
  d.n_filt = m->n_filt;
  d.filt_eo = m->filt_eo;
  d.filt_mo = m->filt_mo;
  d.mats = (const tlm::MatDev *)m->mats_d.p;
  d.exc_field = (const double *)m->exc_field.p;
  d.exc_type = (const int8_t *)m->exc_type.p;
  d.n_exc = m->n_exc_cells;
  d.cell_out = (double *)m->cell_out.p;
  d.cell_cur = (double *)m->cell_cur.p;
  d.out_hist = (const int *)m->out_hist.p;
  d.n_out = m->n_out_cells;
  d.n_hist = m->n_hist;
  d.dl = m->desc.dl;
  d.dt = m->desc.dt;
  d.d_base = (const int *)m->d_base.p;
  d.wrap = m->wrap;
  d.tx_pad = m->tx_pad;
  return d;
}

tlm::FaceDev face_dev(Mesh *m) {
  tlm::FaceDev f{};
  f.face = (const int4 *)m->faces.p;
  f.face_io = (const int2 *)m->face_io.p;
  f.hs = (const double4 *)m->face_hs.p;
  f.n_faces = (int)m->f_cx.size();
  for (int i = 0; i < 3; i++) {
    f.Ei[i] = m->hs_Ei[i];
    f.Hi[i] = m->hs_Hi[i];
  }
  f.offset_min = m->hs_offset_min;
  f.c = m->hs_c;
  f.dt = m->desc.dt;
  f.dl = m->desc.dl;
  f.value_face = (const double *)m->value_face.p;
  f.n_timesteps = m->desc.n_timesteps;
  f.face_field = (double *)m->face_field.p;
  f.face_src = (const int2 *)m->face_src.p;
  f.pt_field = (const double *)m->fpt_field_d.p;
  f.pt_type = (const int8_t *)m->fpt_type_d.p;
  f.n_pt_rows = m->n_pt_rows;
  f.mat = (const int8_t *)m->face_mat_d.p;
  f.smat = (const int *)m->face_smat_d.p;
  f.tl = (const tlm::ThinLayerDev *)m->thin_d.p;
  f.tl_taps = (double *)m->thin_taps.p;
  return f;
}

tlm::OuterHsDev outer_hs_dev(Mesh *m) {
  tlm::OuterHsDev o{};
  o.face = (const int4 *)m->ohs_face.p;
  o.offset = (const double *)m->ohs_offset.p;
  o.n = m->hs_outer ? m->hs_n : 0;
  for (int i = 0; i < 3; i++) {
    o.Ei[i] = m->hs_Ei[i];
    o.Hi[i] = m->hs_Hi[i];
  }
  o.offset_min = m->hs_offset_min;
  o.c = m->hs_c;
  o.dt = m->desc.dt;
  o.dl = m->desc.dl;
  o.value_face = (const double *)m->value_face.p;
  o.n_timesteps = m->desc.n_timesteps;
  return o;
}

tlm::FarFieldDev far_field_dev(Mesh *m) {
  tlm::FarFieldDev d{};
  d.n_entries = m->ff_entries;
  d.n_ff = (int)m->ff_freq.size();
  d.entry = (const int4 *)m->ff_entry.p;
  d.phasor = (const double2 *)m->ff_phasor.p;
  d.face_field = (const double *)m->face_field.p;
  d.acc = (double2 *)m->ff_acc.p;
  return d;
}

tlm::FaceProbeDev face_probe_dev(Mesh *m) {
  return tlm::FaceProbeDev{(const int4 *)m->fprobe.p, (double *)m->fprobe_rec.p, (int)m->fpr_face.size()};
}

tlm::PowerSurfDev power_surf_dev(Mesh *m) {
  tlm::PowerSurfDev d{};
  d.n_entries = m->ps_entries;
  d.n_ps = (int)m->ps_freq.size();
  d.entry = (const int4 *)m->ps_entry.p;
  d.phasor = (const double2 *)m->ps_phasor.p;
  d.face_field = (const double *)m->face_field.p;
  d.acc = (double2 *)m->ps_acc.p;
  return d;
}

tlm::ModeDev mode_dev(Mesh *m) {
  tlm::ModeDev d{};
  d.n_modes = (int)m->mode_comp.size();
  d.mode = (const int4 *)m->mode_d.p;
  d.face = (const int2 *)m->mode_face.p;
  d.weight = (const double *)m->mode_wd.p;
  d.face_field = (const double *)m->face_field.p;
  d.hist = (double *)m->mode_hist.p;
  return d;
}

tlm::SarDev sar_dev(Mesh *m) {
  tlm::SarDev d{};
  d.n_entries = m->sar_entries;
  d.n_vol = (int)m->sar_freq.size();
  d.dt = m->desc.dt;
  d.entry = (const int2 *)m->sar_entry.p;
  d.phasor = (const double2 *)m->sar_phasor.p;
  d.cell_cur = (const double *)m->cell_cur.p;
  d.acc = (double2 *)m->sar_acc.p;
  return d;
}

tlm::OutVolDev out_vol_dev(Mesh *m) {
  tlm::OutVolDev d{};
  d.n_vol = (int)m->ovol_gate.size() / 5;
  d.vol = (const tlm::OVolDev *)m->ovol_dev.p;
  d.cells = (const int *)m->ovol_cells.p;
  d.cell_cur = (const double *)m->cell_cur.p;
  d.hist = (double *)m->ovol_hist.p;
  return d;
}

tlm::RcsDev rcs_dev(Mesh *m) {
  tlm::RcsDev d{};
  d.n_faces = (int)m->rcs_fout.size();
  d.n_points = m->rcs_points;
  d.npc = m->rcs_npc;
  d.offset = m->rcs_offset;
  d.ct = cos(m->rcs_theta); d.st = sin(m->rcs_theta);
  d.cp = cos(m->rcs_phi); d.sp = sin(m->rcs_phi);
  d.dA = m->desc.dl * m->desc.dl;
  d.four_pi = 4.0 * 3.141592653589793;
  d.dl = m->desc.dl;
  d.face = (const int2 *)m->rcs_face.p;
  d.dist = (const double *)m->rcs_dist_d.p;
  d.tc0 = (const double *)m->rcs_tc0.p;
  d.face_field = (const double *)m->face_field.p;
  d.acc = (double *)m->rcs_acc.p;
  return d;
}

tlm::OutSurfDev out_surf_dev(Mesh *m) {
  tlm::OutSurfDev d{};
  d.n_entries = m->osurf_entries;
  d.entry = (const int2 *)m->osurf_entry.p;
  d.pos = (const int2 *)m->osurf_pos.p;
  d.surf = (const tlm::OSurfDev *)m->osurf_dev.p;
  d.face_field = (const double *)m->face_field.p;
  d.hist = (double *)m->osurf_hist.p;
  return d;
}

// Output steps of a surface within 1..n_steps: first..last every interval.
long long osurf_steps(int first, int last, int interval, int n_steps) {
  const int hi = std::min(last, n_steps);
  return hi >= first ? (long long)(hi - first) / interval + 1 : 0;
}

tlm::VolDftDev vol_dft_dev(Mesh *m) {
  tlm::VolDftDev d{};
  d.n_entries = m->vdft_entries;
  d.n_vol = (int)m->vdft_freq.size();
  d.entry = (const int2 *)m->vdft_entry.p;
  d.gate = (const int4 *)m->vdft_gate_d.p;
  d.phasor = (const double2 *)m->vdft_phasor.p;
  d.cell_cur = (const double *)m->cell_cur.p;
  d.acc = (double2 *)m->vdft_acc.p;
  return d;
}

tlm::DftDev dft_dev(Mesh *m) {
  tlm::DftDev d{};
  d.n_entries = m->dft_entries;
  d.n_dft = m->n_dft;
  d.entry = (const int4 *)m->dft_entry.p;
  d.phasor = (const double2 *)m->dft_phasor.p;
  d.face_field = (const double *)m->face_field.p;
  d.acc = (double2 *)m->dft_acc.p;
  return d;
}

// Build and upload all device tables.
// The thicknesses of the box shell that the PML cells form, read off their
// (traversal-ordered, packed) positions, and checked cell by cell; .on = 0
// when the cells are not such a shell (the kernels then load positions).
tlm::PmlShell detect_pml_shell(const std::vector<unsigned long long> &pos, int nx, int ny, int nz) {
  tlm::PmlShell h{};
  if (pos.empty() || (long long)nx * ny > (1ll << 30) || pos.size() > (size_t)INT32_MAX) return h;
  auto X = [](unsigned long long p) { return (int)(p & 0x1fffffull); };
  auto Y = [](unsigned long long p) { return (int)((p >> 21) & 0x1fffffull); };
  auto Z = [](unsigned long long p) { return (int)((p >> 42) & 0x1fffffull); };
  // slab thicknesses: leading / trailing z-planes that are entirely PML,
  // then, in the first plane between them, leading / trailing full rows,
  // then the leading / trailing run of x in the first row between those
  std::vector<long long> per_z(nz, 0);
  for (auto p : pos) per_z[Z(p)]++;
  const long long full = (long long)nx * ny;
  int zl = 0, zh = 0;
  while (zl < nz && per_z[zl] == full) zl++;
  while (zh < nz - zl && per_z[nz - 1 - zh] == full) zh++;
  int yl = 0, yh = 0, xl = 0, xh = 0;
  if (zl + zh < nz) {
    const int zm = zl;
    std::vector<int> per_y(ny, 0);
    for (auto p : pos)
      if (Z(p) == zm) per_y[Y(p)]++;
    while (yl < ny && per_y[yl] == nx) yl++;
    while (yh < ny - yl && per_y[ny - 1 - yh] == nx) yh++;
    if (yl + yh < ny) {
      std::vector<char> xin(nx, 0);
      for (auto p : pos)
        if (Z(p) == zm && Y(p) == yl) xin[X(p)] = 1;
      while (xl < nx && xin[xl]) xl++;
      while (xh < nx - xl && xin[nx - 1 - xh]) xh++;
    }
  }
  h.nx = nx; h.ny = ny; h.nz = nz;
  h.xl = xl; h.xh = xh; h.yl = yl; h.yh = yh; h.zl = zl; h.zh = zh;
  h.full = (int)full;
  h.partial = (yl + yh) * nx + (ny - yl - yh) * (xl + xh);
  h.d_full = tlm::make_fast_div(h.full);
  h.d_nx = tlm::make_fast_div(nx);
  h.d_partial = tlm::make_fast_div(h.partial);
  h.d_w = tlm::make_fast_div(xl + xh);
  const long long count = (long long)(zl + zh) * full + (long long)(nz - zl - zh) * h.partial;
  if (count != (long long)pos.size()) return tlm::PmlShell{};
  // the decoder the kernels run must reproduce every listed position
  for (size_t s = 0; s < pos.size(); s++) {
    int x, y, z;
    tlm::pml_shell_pos(h, (int)s, x, y, z);
    if (x != X(pos[s]) || y != Y(pos[s]) || z != Z(pos[s])) return tlm::PmlShell{};
  }
  h.on = 1;
  return h;
}

int finalize(Mesh *m) {
  if (m->finalized) return TLM_OK;
  const auto &D = m->desc;
  const int nx = D.nx, ny = D.ny, nz = D.nz;
  const long long ncell = (long long)nx * ny * nz;
  const int nsteps = D.n_timesteps;
  CK(cudaSetDevice(D.device));
  if (!m->have_cells) {
    m->cell_code.assign(ncell, 0);
    m->n_special = 0;
  }
  // ---- validate cross references
  for (int s = 0; s < m->n_special; s++) {
    const int mat = m->sp_material[s], pml = m->sp_pml[s];
    if (mat < 0 || mat > (int)m->mats.size()) return fail(TLM_E_BADARG, "special cell %d: material %d out of range", s + 1, mat);
    if (pml < 0 || pml > m->n_pml_cells) return fail(TLM_E_BADARG, "special cell %d: PML cell %d out of range", s + 1, pml);
    if (pml && mat) {
      const int type = m->mats[mat - 1].type;
      if (type == 1 || type == 2) return fail(TLM_E_UNSUPPORTED, "PEC/PMC volume material in PML (scatter.F90:559-567)");
      if (m->pml_sigma.empty())
        return fail(TLM_E_BADARG, "PML cell %d lies in material %d: tlm_gpu_set_pml_sigma is required", pml, mat);
    }
    if (pml && m->sp_exc[s]) return fail(TLM_E_UNSUPPORTED, "Excitation intersects PML (set_update_codes.F90:347-354)");
  }
  // ---- special cell tables: masks, prefix bases, records
  const int VEC = m->fp64 ? 2 : 4;
  (void)VEC;
  const int per_plane = ny * m->Px;
  const int segs_pp = (per_plane + 31) / 32;
  std::vector<uint32_t> mask((size_t)segs_pp * nz, 0u), base((size_t)segs_pp * nz, 0u);
  std::vector<int4> rec, pos;
  rec.reserve(m->n_special + 1);
  pos.reserve(m->n_special + 1);
  std::vector<unsigned long long> pml_pos;
  std::vector<uint16_t> pml_par;
  std::vector<int2> pml_out;
  std::vector<int4> pmm_pos;
  std::vector<int2> pmm_parmat;
  pml_pos.reserve(m->n_pml_cells + 1);
  pml_par.reserve(m->n_pml_cells + 1);
  int mask_count = 0;
  // filter storage per dispersive cell (allocate_volume_material_filter_data)
  int eo = 0, mo = 0;
  for (auto &md : m->mats) {
    if (md.type == 3) {
      if (md.eps_exists) eo = std::max(eo, md.eps_order);
      if (md.mu_exists) mo = std::max(mo, md.mu_order);
    }
  }
  m->filt_eo = eo;
  m->filt_mo = mo;
  int n_filt = 0, exc_no = 0, out_no = 0;
  long long cell = 0;
  uint32_t running = 0;
  for (int z = 0; z < nz; z++) {
    for (int y = 0; y < ny; y++) {
      for (int x = 0; x < nx; x++, cell++) {
        const int code = m->cell_code[cell];
        if (code == 0) continue;
        if (code < 0 || code > m->n_special) return fail(TLM_E_BADARG, "cell_centre_update_code out of range at cell %lld", cell + 1);
        const int s = code - 1;
        const int e = y * m->Px + x;
        const size_t sg = (size_t)z * segs_pp + (e >> 5);
        mask[sg] |= 1u << (e & 31);
        mask_count++;
        int flags = 0;
        const int mat = m->sp_material[s];
        int4 r{0, -1, -1, -1};
        if (m->sp_pml[s]) {
          // PML cells go to the packed PML list; PML cell numbers follow traversal order
          const int pidx = m->sp_pml[s] - 1;
          if (pidx != (int)pml_pos.size())
            return fail(TLM_E_BADARG, "PML cell numbers must follow (cz,cy,cx) traversal order (cell %lld)", cell + 1);
          const int par = m->pml_cell_param[pidx];
          if (par < 1 || par > m->n_pml_params)
            return fail(TLM_E_BADARG, "PML cell %d: parameter %d out of range", pidx + 1, par);
          if (par > tlm::kPmlOutputFlag - 1)  // bit 15 of the packed index is the output flag
            return fail(TLM_E_UNSUPPORTED, "more than %d PML parameter rows", tlm::kPmlOutputFlag - 1);
          unsigned long long pk = (unsigned long long)x | ((unsigned long long)y << 21) | ((unsigned long long)z << 42);
          if (mat) {  // PML cell in a volume material: own list, own kernel
            pmm_pos.push_back(int4{x, y, z, m->sp_out[s] ? out_no++ : -1});
            pmm_parmat.push_back(int2{par - 1, mat});
            pml_pos.push_back(pk);
            pml_par.push_back(tlm::kPmlMaterialSlot);
            continue;
          }
          int pw = par - 1;
          if (m->sp_out[s]) {
            pk |= 1ull << 63;
            pml_out.push_back(int2{pidx, out_no++});
            pw |= tlm::kPmlOutputFlag;
          }
          pml_pos.push_back(pk);
          pml_par.push_back((uint16_t)pw);
          continue;
        } else {
          if (mat) {
            flags |= tlm::SP_MAT;
            if (m->mats[mat - 1].type == 3) r.y = (int)rec.size();  // taps slot = record index
          }
          if (m->sp_exc[s]) {
            flags |= tlm::SP_EXC;
            r.z = exc_no++;
          }
        }
        if (m->sp_out[s]) {
          flags |= tlm::SP_OUT;
          r.w = out_no++;
        }
        r.x = flags | (mat << 8);
        rec.push_back(r);
        pos.push_back(int4{x, y, z, 0});
      }
    }
  }
  // the records are pushed in traversal order, which is also mask order
  // within (z, e): rebuild bases as exclusive prefix counts of mask bits
  running = 0;
  for (size_t i = 0; i < mask.size(); i++) {
    base[i] = running;
    running += __builtin_popcount(mask[i]);
  }
  if ((int)running != mask_count || (int)(rec.size() + pml_pos.size()) != mask_count)
    return fail(TLM_E_BADARG, "special cell count mismatch");
  if ((int)pml_pos.size() != m->n_pml_cells) return fail(TLM_E_BADARG, "PML cells: %zu flagged, %d declared", pml_pos.size(), m->n_pml_cells);
  if (nx >= (1 << 21) || ny >= (1 << 21) || nz >= (1 << 21)) return fail(TLM_E_BADARG, "mesh too large for packed positions");
  m->n_pml_list = (int)pml_pos.size();
  m->pml_shell = detect_pml_shell(pml_pos, nx, ny, nz);
  if (const char *e = getenv("TLM_PML_SHELL"))  // "0": load positions even for a shell
    if (e[0] == '0') m->pml_shell = tlm::PmlShell{};
  m->n_pmm = (int)pmm_pos.size();
  if (m->n_pmm) {
    int rc2;
    std::vector<double> sg((size_t)m->n_pml_params * 4, 0.0);
    for (int i = 0; i < m->n_pml_params; i++)
      for (int k = 0; k < 3; k++) sg[(size_t)i * 4 + k] = m->pml_sigma[(size_t)i * 3 + k];
    if ((rc2 = upload(m, m->pmm_pos, pmm_pos)) || (rc2 = upload(m, m->pmm_parmat, pmm_parmat)) ||
        (rc2 = upload(m, m->pmm_sigma, sg)) ||
        (rc2 = dalloc(m, m->pmm_state, (size_t)tlm::kPmmState * m->n_pmm * sizeof(double))))
      return rc2;
    CK(cudaMemset(m->pmm_state.p, 0, m->pmm_state.bytes));  // allocate_PML_material_data: all zero
  }
  m->n_pml_out = (int)pml_out.size();
  if (pml_out.empty()) pml_out.resize(1);
  {
    int rc2;
    pml_pos.resize(pml_pos.size() + 8, 0ull);  // 64 bytes of padding for the widened L2 prefetch
    pml_par.resize(pml_par.size() + 128, 0);    // 256 bytes of padding for the index L2 prefetch
    if ((rc2 = upload(m, m->pml_pos, pml_pos)) || (rc2 = upload(m, m->pml_par16, pml_par)) ||
        (rc2 = upload(m, m->pml_outmap, pml_out)))
      return rc2;
  }
  if (exc_no != m->n_exc_cells) return fail(TLM_E_BADARG, "excitation cells: %d flagged, %d declared", exc_no, m->n_exc_cells);
  if (out_no != m->n_out_cells) return fail(TLM_E_BADARG, "output cells: %d flagged, %d declared", out_no, m->n_out_cells);
  n_filt = (int)rec.size();  // one tap slot per record (special_cell loads taps by record index)
  m->n_filt = n_filt;
  m->n_sp_dev = (int)rec.size();
  int rc;
  m->host_mask = mask;
  if ((rc = upload(m, m->seg_mask, mask)) || (rc = upload(m, m->seg_base, base)) || (rc = upload(m, m->sp_rec, rec)) ||
      (rc = upload(m, m->sp_pos, pos)))
    return rc;
  // ---- links (zeroed, allocate_mesh.F90:120)
  const size_t esz = m->fp64 ? 8 : 4;
  if ((rc = dalloc(m, m->links, 2 * 12 * (size_t)m->plane * esz))) return rc;
  CK(cudaMemset(m->links.p, 0, m->links.bytes));
  // ---- PML
  const size_t pesz = m->fp64 ? sizeof(tlm::PmlTypes<double>::state) : sizeof(tlm::PmlTypes<float>::state);
  if ((rc = dalloc(m, m->pml_state, tlm::pml_state_elems(std::max(m->n_pml_cells, 1)) * pesz + 64))) return rc;
  CK(cudaMemset(m->pml_state.p, 0, m->pml_state.bytes));
  {
    std::vector<double> par((size_t)std::max(m->n_pml_params, 1) * 16, 0.0);
    for (int i = 0; i < m->n_pml_params; i++)
      for (int k = 0; k < 15; k++) par[(size_t)i * 16 + k] = m->pml_params[(size_t)i * 15 + k];
    if ((rc = upload(m, m->pml_par, par))) return rc;
    // the parameter rows by distance class, where every cell's row is its
    // class's (TLM_PML_CLASS=0 turns the class path off)
    m->pml_by_class = false;
    const char *ce = getenv("TLM_PML_CLASS");
    if (m->pml_shell.on && m->n_pml_list && !(ce && ce[0] == '0')) {
      const tlm::PmlShell &h = m->pml_shell;
      const size_t ncls = (size_t)(h.xl + h.xh + 1) * (h.yl + h.yh + 1) * (h.zl + h.zh + 1);
      std::vector<int> row_of(ncls, -1);
      bool ok = true;
      for (int s2 = 0; s2 < m->n_pml_list && ok; s2++) {
        if (pml_par[s2] == tlm::kPmlMaterialSlot) continue;
        const int row = pml_par[s2] & (tlm::kPmlOutputFlag - 1);
        int x, y, z;
        tlm::pml_shell_pos(h, s2, x, y, z);
        const int c = tlm::pml_class(h, x, y, z);
        if (c < 0 || (size_t)c >= ncls) ok = false;
        else if (row_of[c] < 0) row_of[c] = row;
        else if (row_of[c] != row) ok = false;
      }
      if (ok) {
        std::vector<double> cp(ncls * 16, 0.0);
        for (size_t c = 0; c < ncls; c++)
          if (row_of[c] >= 0)
            for (int k = 0; k < 16; k++) cp[c * 16 + k] = par[(size_t)row_of[c] * 16 + k];
        if ((rc = upload(m, m->pml_cls_par, cp))) return rc;
        m->pml_by_class = true;
      }
    }
  }
  if ((rc = dalloc(m, m->pml_ixt, (size_t)std::max(m->n_out_cells, 1) * 3 * pesz))) return rc;
  CK(cudaMemset(m->pml_ixt.p, 0, m->pml_ixt.bytes));
  // ---- filters + materials
  const size_t J = 3 * (size_t)(eo + mo);
  if ((rc = dalloc(m, m->filt, std::max<size_t>(J, 1) * std::max(n_filt, 1) * sizeof(double)))) return rc;
  CK(cudaMemset(m->filt.p, 0, m->filt.bytes));
  {
    std::vector<tlm::MatDev> md = m->mats;
    if (md.empty()) md.resize(1);
    if ((rc = upload(m, m->mats_d, md))) return rc;
  }
  // ---- per-step cell excitation (excitation() + Point_excitation)
  {
    const int ne = m->n_exc_cells;
    std::vector<double> field((size_t)std::max(ne, 1) * 9 * nsteps, 0.0);
    std::vector<int8_t> type((size_t)std::max(ne, 1) * 6, 1);
    for (size_t p = 0; p < m->pt_cell.size(); p++) {
      const int c = m->pt_cell[p] - 1, comp = m->pt_comp[p] - 1, fn = m->pt_fn[p] - 1;
      if (c < 0 || c >= ne || comp < 0 || comp >= 9 || fn < 0 || fn >= m->n_fn)
        return fail(TLM_E_BADARG, "point excitation %zu: bad cell/component/function", p + 1);
      if (comp < 6) type[(size_t)c * 6 + comp] = (int8_t)m->pt_type[p];
    }
    for (int t = 0; t < nsteps; t++) {
      double *row = field.data() + (size_t)t * std::max(ne, 1) * 9;
      for (size_t p = 0; p < m->pt_cell.size(); p++) {
        const int c = m->pt_cell[p] - 1, comp = m->pt_comp[p] - 1, fn = m->pt_fn[p] - 1;
        const double v = t < m->n_fn_steps ? m->fn_value[(size_t)fn * m->n_fn_steps + t] : 0.0;
        row[(size_t)c * 9 + comp] = row[(size_t)c * 9 + comp] + v;
      }
    }
    if ((rc = upload(m, m->exc_field, field)) || (rc = upload(m, m->exc_type, type))) return rc;
  }
  // ---- cell outputs: the current-step rows of all of them, the time series
  // of those that keep one
  {
    const int no = m->n_out_cells;
    if (!m->out_keep.empty() && (int)m->out_keep.size() != no)
      return fail(TLM_E_BADARG, "output series flags: %zu given for %d output cells", m->out_keep.size(), no);
    std::vector<int32_t> slot(std::max(no, 1), -1);
    int nh = 0;
    for (int i = 0; i < no; i++)
      if (m->out_keep.empty() || m->out_keep[i]) slot[i] = nh++;
    m->n_hist = nh;
    if ((rc = upload(m, m->out_hist, slot))) return rc;
    if ((rc = dalloc(m, m->cell_cur, (size_t)std::max(no, 1) * 6 * sizeof(double)))) return rc;
    CK(cudaMemset(m->cell_cur.p, 0, m->cell_cur.bytes));
    if ((rc = dalloc(m, m->cell_out, (size_t)std::max(nh, 1) * 6 * nsteps * sizeof(double)))) return rc;
    CK(cudaMemset(m->cell_out.p, 0, m->cell_out.bytes));
  }
  // ---- frequency output volumes
  {
    const int nv = (int)m->vdft_freq.size();
    std::vector<int2> ent;
    std::vector<int4> gate(std::max(nv, 1), int4{1, 0, 1, 1});
    for (int v = 0; v < nv; v++) {
      const int *g = &m->vdft_gate[(size_t)v * 4];
      if (g[3] < 1 || g[3] > 6) return fail(TLM_E_BADARG, "output volume %d: component %d is not Ex..Hz", v + 1, g[3]);
      if (g[2] < 1) return fail(TLM_E_BADARG, "output volume %d: timestep interval must be >= 1", v + 1);
      gate[v] = int4{g[0], g[1], g[2], g[3]};
      for (int k = m->vdft_ptr[v]; k < m->vdft_ptr[v + 1]; k++) {
        const int o = m->vdft_out[k];
        if (o < 1 || o > m->n_out_cells) return fail(TLM_E_BADARG, "output volume %d: output cell %d out of range", v + 1, o);
        ent.push_back(int2{v, o - 1});
      }
    }
    m->vdft_entries = (int)ent.size();
    if (ent.empty()) ent.resize(1);
    std::vector<double2> ph((size_t)std::max(nv, 1) * nsteps, double2{0, 0});
    const double pi = 3.141592653589793;
    for (int t = 0; t < nsteps; t++) {
      const double time = (double)t * D.dt;  // (timestep-1)*dt: cell outputs come before the half step
      for (int v = 0; v < nv; v++) {
        const double arg = -2.0 * pi * m->vdft_freq[v] * time;
        ph[(size_t)t * nv + v] = double2{cos(arg), sin(arg)};
      }
    }
    if ((rc = upload(m, m->vdft_entry, ent)) || (rc = upload(m, m->vdft_gate_d, gate)) ||
        (rc = upload(m, m->vdft_phasor, ph)))
      return rc;
    if ((rc = dalloc(m, m->vdft_acc, ent.size() * sizeof(double2)))) return rc;
    CK(cudaMemset(m->vdft_acc.p, 0, m->vdft_acc.bytes));
  }
  // ---- special faces
  {
    const int nf = (int)m->f_cx.size();
    std::vector<int4> fc(std::max(nf, 1));
    std::vector<int2> io(std::max(nf, 1));
    std::vector<double4> hs(std::max(nf, 1), double4{0, 0, 0, 0});
    std::vector<int> exc_to_face(m->n_exc_faces + 1, -1);
    for (int f = 0; f < nf; f++) {
      const int x = m->f_cx[f] - 1, y = m->f_cy[f] - 1, z = m->f_cz[f] - 1, d = m->f_dir[f];
      if (d < 1 || d > 3 || x < 0 || x >= nx || y < 0 || y >= ny || z < 0 || z >= nz)
        return fail(TLM_E_BADARG, "special face %d out of range", f + 1);
      if ((d == 1 && x == 0) || (d == 2 && y == 0) || (d == 3 && z == 0))
        return fail(TLM_E_BADARG, "special face %d lies on the outer boundary", f + 1);
      fc[f] = int4{x, y, z, d};
      io[f] = int2{m->f_exc[f] ? m->f_exc[f] - 1 : -1, m->f_out[f] ? m->f_out[f] - 1 : -1};
      if (m->f_exc[f]) {
        if (m->f_exc[f] > m->n_exc_faces) return fail(TLM_E_BADARG, "face excitation number out of range");
        exc_to_face[m->f_exc[f]] = f;
      }
      if (m->f_out[f] > m->n_out_faces) return fail(TLM_E_BADARG, "face output number out of range");
    }
    if (!m->f_mat.empty() && (int)m->f_mat.size() != nf)
      return fail(TLM_E_BADARG, "face materials: %zu given for %d special faces", m->f_mat.size(), nf);
    std::vector<int8_t> fmat(std::max(nf, 1), 0);
    if (!m->f_smat.empty() && (int)m->f_smat.size() != nf)
      return fail(TLM_E_BADARG, "face thin layers: %zu given for %d special faces", m->f_smat.size(), nf);
    std::vector<int> fsmat(std::max(nf, 1), 0);
    for (int f = 0; f < (int)m->f_mat.size(); f++) {
      const int t = m->f_mat[f];
      if (t != 0 && t != 1 && t != 2 && t != 3 && t != 4)
        return fail(TLM_E_UNSUPPORTED,
                    "special face %d: surface material type %d (only PEC 1, PMC 2, thin layer 3, free space 4)", f + 1, t);
      fmat[f] = (int8_t)t;
      const int sm = m->f_smat.empty() ? 0 : m->f_smat[f];
      if ((t == 3) != (sm != 0))
        return fail(TLM_E_BADARG, "special face %d: a thin layer needs material type 3 and a thin-layer material", f + 1);
      if (sm && std::abs(sm) > (int)m->thin.size())
        return fail(TLM_E_BADARG, "special face %d: thin-layer material %d is not defined", f + 1, std::abs(sm));
      fsmat[f] = sm;
    }
    if (m->f_mat.empty())
      for (int f = 0; f < (int)m->f_smat.size(); f++)
        if (m->f_smat[f]) return fail(TLM_E_BADARG, "special face %d: a thin layer needs material type 3", f + 1);
    {
      std::vector<tlm::ThinLayerDev> tl = m->thin;
      if (tl.empty()) tl.resize(1);
      if ((rc = upload(m, m->face_mat_d, fmat)) || (rc = upload(m, m->face_smat_d, fsmat)) ||
          (rc = upload(m, m->thin_d, tl)) ||
          (rc = dalloc(m, m->thin_taps, (size_t)std::max(nf, 1) * 8 * tlm::kMaxOrder * sizeof(double))))
        return rc;
      CK(cudaMemset(m->thin_taps.p, 0, m->thin_taps.bytes));  // allocate_Zfilter_response: w = 0
    }
    std::vector<int> covered(m->n_exc_faces + 1, 0);
    std::vector<int2> src(std::max(nf, 1), int2{0, -1});
    for (int h = 0; h < (m->hs_outer ? 0 : m->hs_n); h++) {
      const int e = m->hs_face_exc[h];
      if (e < 1 || e > m->n_exc_faces || exc_to_face[e] < 0) return fail(TLM_E_BADARG, "Huygens patch %d: bad face excitation number", h + 1);
      if (covered[e]++) return fail(TLM_E_UNSUPPORTED, "two Huygens patches on one face");
      hs[exc_to_face[e]] = double4{m->hs_offset[h], (double)m->hs_norm[3 * h], (double)m->hs_norm[3 * h + 1],
                                   (double)m->hs_norm[3 * h + 2]};
      src[exc_to_face[e]].x = 1;
    }
    // face point sources: one row of summed fields per excitation face that
    // has any, side 1 then side 2, tabulated for every step from the
    // functions' value_face
    std::vector<int> row_of(m->n_exc_faces + 1, -1);
    const int npt = (int)m->fpt_face.size();
    if (!m->fpt_side.empty() && (int)m->fpt_side.size() != npt)
      return fail(TLM_E_BADARG, "face source sides: %d given for %d face sources", (int)m->fpt_side.size(), npt);
    if (!m->fpt_scale.empty() && (int)m->fpt_scale.size() != npt)
      return fail(TLM_E_BADARG, "face source scales: %d given for %d face sources", (int)m->fpt_scale.size(), npt);
    m->n_pt_rows = 0;
    for (int e = 0; e < npt; e++) {
      const int fe = m->fpt_face[e], comp = m->fpt_comp[e], fn = m->fpt_fn[e], ty = m->fpt_type[e];
      if (fe < 1 || fe > m->n_exc_faces || exc_to_face[fe] < 0) return fail(TLM_E_BADARG, "face point source %d: bad face excitation number", e + 1);
      if (comp < 1 || comp > 12) return fail(TLM_E_BADARG, "face point source %d: component %d out of range", e + 1, comp);
      if (fn < 1 || fn > m->n_fn) return fail(TLM_E_BADARG, "face point source %d: function out of range", e + 1);
      if (ty != 0 && ty != 1) return fail(TLM_E_BADARG, "face point source %d: source type must be 0 (hard) or 1 (soft)", e + 1);
      if (!m->fpt_side.empty() && (m->fpt_side[e] < 0 || m->fpt_side[e] > 2))
        return fail(TLM_E_BADARG, "face point source %d: side must be 0 (both), 1 or 2", e + 1);
      if (row_of[fe] < 0) row_of[fe] = m->n_pt_rows++;
      covered[fe]++;
    }
    for (int e = 1; e <= m->n_exc_faces; e++) {
      if (!covered[e]) return fail(TLM_E_BADARG, "face excitation %d has neither a Huygens patch nor a point source", e);
      if (row_of[e] >= 0) src[exc_to_face[e]].y = row_of[e];
    }
    {
      const int R = std::max(m->n_pt_rows, 1);
      std::vector<double> ptf((size_t)nsteps * R * 24, 0.0);
      std::vector<int8_t> ptt((size_t)R * 6, 1);  // set_update_codes.F90:593, soft
      for (int e = 0; e < npt; e++) {
        const int r = row_of[m->fpt_face[e]], c = m->fpt_comp[e] - 1, fn = m->fpt_fn[e] - 1;
        const int only = m->fpt_side.empty() ? 0 : m->fpt_side[e];
        const bool scaled = !m->fpt_scale.empty();
        const double sc = scaled ? m->fpt_scale[e] : 1.0;
        for (int sd = 0; sd < 2; sd++) {
          if (only && sd != only - 1) continue;
          for (int t = 0; t < nsteps && t < m->n_fn_steps; t++) {
            const double fv = m->fn_value_face[(size_t)fn * m->n_fn_steps + t];
            double &v = ptf[((size_t)t * R + r) * 24 + sd * 12 + c];
            v = v + (scaled ? sc * fv : fv);  // Mode_excitation: face_excitation_field + mode_field*value
          }
        }
        // connect reads side 1's source types on both sides
        if (c < 6 && only != 2) ptt[(size_t)r * 6 + c] = (int8_t)m->fpt_type[e];
      }
      if ((rc = upload(m, m->fpt_field_d, ptf)) || (rc = upload(m, m->fpt_type_d, ptt)) || (rc = upload(m, m->face_src, src)))
        return rc;
    }
    // face output points
    {
      const int nq = (int)m->fpr_face.size();
      std::vector<int4> pq(std::max(nq, 1), int4{0, 0, 0, 0});
      for (int q = 0; q < nq; q++) {
        if (m->fpr_face[q] < 1 || m->fpr_face[q] > m->n_out_faces || m->fpr_side[q] < 1 || m->fpr_side[q] > 2 ||
            m->fpr_comp[q] < 1 || m->fpr_comp[q] > 6)
          return fail(TLM_E_BADARG, "face output point %d: face, side or component out of range", q + 1);
        pq[q] = int4{m->fpr_face[q] - 1, m->fpr_side[q] - 1, m->fpr_comp[q] - 1, 0};
      }
      if ((rc = upload(m, m->fprobe, pq)) ||
          (rc = dalloc(m, m->fprobe_rec, (size_t)std::max(nq, 1) * nsteps * sizeof(double))))
        return rc;
      CK(cudaMemset(m->fprobe_rec.p, 0, m->fprobe_rec.bytes));
    }
    if ((rc = upload(m, m->faces, fc)) || (rc = upload(m, m->face_io, io)) || (rc = upload(m, m->face_hs, hs))) return rc;
    std::vector<double> vf(std::max(nsteps, 1), 0.0);
    if (m->hs_n) {
      if (m->hs_fn < 1 || m->hs_fn > m->n_fn) return fail(TLM_E_BADARG, "Huygens function number out of range");
      for (int t = 0; t < nsteps && t < m->n_fn_steps; t++) vf[t] = m->fn_value_face[(size_t)(m->hs_fn - 1) * m->n_fn_steps + t];
    }
    if ((rc = upload(m, m->value_face, vf))) return rc;
    // outer-boundary Huygens patches
    if (m->hs_outer && m->wrap)  // its terms would go to the slots before the wrap moves them
      return fail(TLM_E_UNSUPPORTED, "an outer-boundary Huygens surface with wrapping boundaries");
    if (m->hs_outer) {
      std::vector<int4> of(std::max(m->hs_n, 1));
      for (int h = 0; h < m->hs_n; h++) {
        const int x = m->hs_cell[4 * h] - 1, y = m->hs_cell[4 * h + 1] - 1, z = m->hs_cell[4 * h + 2] - 1;
        const int code = m->hs_cell[4 * h + 3];
        const bool ok = x >= 0 && x < nx && y >= 0 && y < ny && z >= 0 && z < nz && code >= 1 && code <= 6 &&
                        ((code == 1 && x == 0) || (code == 4 && x == nx - 1) || (code == 2 && y == 0) ||
                         (code == 5 && y == ny - 1) || (code == 3 && z == 0) || (code == 6 && z == nz - 1));
        if (!ok) return fail(TLM_E_BADARG, "outer Huygens patch %d is not a boundary face of the mesh", h + 1);
        of[h] = int4{x, y, z, code};
      }
      std::vector<double> oo(m->hs_offset.begin(), m->hs_offset.end());
      if (oo.empty()) oo.resize(1);
      if ((rc = upload(m, m->ohs_face, of)) || (rc = upload(m, m->ohs_offset, oo))) return rc;
    }
    if ((rc = dalloc(m, m->face_field, (size_t)std::max(m->n_out_faces, 1) * 12 * sizeof(double)))) return rc;
    CK(cudaMemset(m->face_field.p, 0, m->face_field.bytes));
  }
  // ---- DFT
  {
    std::vector<int4> ent;
    for (int d = 0; d < m->n_dft; d++) {
      for (int k = m->dft_ptr[d]; k < m->dft_ptr[d + 1]; k++) {
        const int fo = m->dft_fout[k];
        if (fo < 1 || fo > m->n_out_faces) return fail(TLM_E_BADARG, "DFT face output number out of range");
        const int comp = m->dft_comp[d];
        if (comp < 1 || comp > 9) return fail(TLM_E_BADARG, "DFT component out of range");
        ent.push_back(int4{d, fo - 1, m->dft_fcode[k], comp});
      }
    }
    m->dft_entries = (int)ent.size();
    if (ent.empty()) ent.resize(1);
    std::vector<double2> ph((size_t)std::max(m->n_dft, 1) * nsteps, double2{0, 0});
    const double pi = 3.141592653589793;
    for (int t = 0; t < nsteps; t++) {
      double time = (double)t * D.dt;  // (timestep-1)*dt
      time = time + D.dt / 2.0;
      for (int d = 0; d < m->n_dft; d++) {
        // get_output_flag (output.F90:564-598): a step outside the
        // surface's output steps adds value * 0
        if (!m->dft_gate.empty()) {
          const int ts = t + 1, f = m->dft_gate[3 * d], l = m->dft_gate[3 * d + 1], iv = m->dft_gate[3 * d + 2];
          if (ts < f || ts > l || (ts - f) % iv != 0) continue;
        }
        const double arg = -2.0 * pi * m->dft_freq[d] * time;
        ph[(size_t)t * m->n_dft + d] = double2{cos(arg), sin(arg)};
      }
    }
    if ((rc = upload(m, m->dft_entry, ent)) || (rc = upload(m, m->dft_phasor, ph))) return rc;
    if ((rc = dalloc(m, m->dft_acc, ent.size() * sizeof(double2)))) return rc;
    CK(cudaMemset(m->dft_acc.p, 0, m->dft_acc.bytes));
  }
  // ---- far-field surfaces
  {
    const int nff = (int)m->ff_freq.size();
    std::vector<int4> ent;
    for (int d = 0; d < nff; d++) {
      for (int k = m->ff_ptr[d]; k < m->ff_ptr[d + 1]; k++) {
        const int fo = m->ff_fout[k], code = m->ff_fcode[k];
        if (fo < 1 || fo > m->n_out_faces) return fail(TLM_E_BADARG, "far-field face output number out of range");
        if (code < 1 || code > 6) return fail(TLM_E_BADARG, "far-field face code out of range");
        ent.push_back(int4{d, fo - 1, code, 0});
      }
    }
    m->ff_entries = (int)ent.size();
    if (ent.empty()) ent.resize(1);
    std::vector<double2> ph((size_t)std::max(nff, 1) * nsteps, double2{0, 0});
    const double pi = 3.141592653589793;
    for (int t = 0; t < nsteps; t++) {
      double time = (double)t * D.dt;  // (timestep-1)*dt
      time = time + D.dt / 2.0;
      for (int d = 0; d < nff; d++) {
        const double arg = -2.0 * pi * m->ff_freq[d] * time;
        ph[(size_t)t * nff + d] = double2{cos(arg) * D.dt, sin(arg) * D.dt};
      }
    }
    if ((rc = upload(m, m->ff_entry, ent)) || (rc = upload(m, m->ff_phasor, ph))) return rc;
    if ((rc = dalloc(m, m->ff_acc, ent.size() * 6 * sizeof(double2)))) return rc;
    CK(cudaMemset(m->ff_acc.p, 0, m->ff_acc.bytes));
  }
  // ---- time-domain output surfaces
  {
    const int ns = (int)m->osurf_gate.size() / 5;
    std::vector<int2> ent, pos;
    std::vector<tlm::OSurfDev> sd(std::max(ns, 1));
    size_t off = 0;
    for (int v = 0; v < ns; v++) {
      const int *g = &m->osurf_gate[(size_t)v * 5];
      const int comp = g[3];
      if (!((comp >= 1 && comp <= 9) || (comp >= 13 && comp <= 15)))
        return fail(TLM_E_BADARG, "output surface %d: component %d is not E, H, J or a magnitude", v + 1, comp);
      if (g[0] < 1 || g[2] < 1) return fail(TLM_E_BADARG, "output surface %d: first step and interval must be >= 1", v + 1);
      if (g[4] != 0 && g[4] != 1) return fail(TLM_E_BADARG, "output surface %d: both-sides flag must be 0 or 1", v + 1);
      const int nf = m->osurf_ptr[v + 1] - m->osurf_ptr[v];
      sd[v] = tlm::OSurfDev{int4{g[0], g[1], g[2], comp}, g[4], nf, (long long)off};
      for (int k = m->osurf_ptr[v]; k < m->osurf_ptr[v + 1]; k++) {
        const int fo = m->osurf_fout[k], code = m->osurf_fcode[k];
        if (fo < 1 || fo > m->n_out_faces) return fail(TLM_E_BADARG, "output surface %d: face output number out of range", v + 1);
        if (code < 1 || code > 6) return fail(TLM_E_BADARG, "output surface %d: face code out of range", v + 1);
        ent.push_back(int2{v, fo - 1});
        pos.push_back(int2{code, k - m->osurf_ptr[v]});
      }
      off += (size_t)osurf_steps(g[0], g[1], g[2], nsteps) * (size_t)nf;
    }
    m->osurf_entries = (int)ent.size();
    m->osurf_hist_len = off;
    if (ent.empty()) { ent.resize(1); pos.resize(1); }
    if ((rc = upload(m, m->osurf_entry, ent)) || (rc = upload(m, m->osurf_pos, pos)) || (rc = upload(m, m->osurf_dev, sd)))
      return rc;
    if ((rc = dalloc(m, m->osurf_hist, std::max<size_t>(off, 1) * sizeof(double)))) return rc;
    CK(cudaMemset(m->osurf_hist.p, 0, m->osurf_hist.bytes));
  }
  // ---- frequency-domain power surfaces
  {
    const int np_ = (int)m->ps_freq.size();
    std::vector<int4> ent;
    for (int v = 0; v < np_; v++)
      for (int k = m->ps_ptr[v]; k < m->ps_ptr[v + 1]; k++) {
        const int fo = m->ps_fout[k], code = m->ps_fcode[k];
        if (fo < 1 || fo > m->n_out_faces) return fail(TLM_E_BADARG, "power surface %d: face output number out of range", v + 1);
        if (code < 1 || code > 6) return fail(TLM_E_BADARG, "power surface %d: face code out of range", v + 1);
        ent.push_back(int4{v, fo - 1, code, 0});
      }
    m->ps_entries = (int)ent.size();
    if (ent.empty()) ent.resize(1);
    std::vector<double2> ph((size_t)std::max(np_, 1) * nsteps, double2{0, 0});
    const double pi = 3.141592653589793;
    for (int t = 0; t < nsteps; t++) {
      double time = (double)t * D.dt;  // (timestep-1)*dt, then the half step of the face outputs
      time = time + D.dt / 2.0;
      for (int v = 0; v < np_; v++) {
        const double arg = -2.0 * pi * m->ps_freq[v] * time;
        ph[(size_t)t * np_ + v] = double2{cos(arg), sin(arg)};
      }
    }
    if ((rc = upload(m, m->ps_entry, ent)) || (rc = upload(m, m->ps_phasor, ph))) return rc;
    if ((rc = dalloc(m, m->ps_acc, ent.size() * 4 * sizeof(double2)))) return rc;
    CK(cudaMemset(m->ps_acc.p, 0, m->ps_acc.bytes));
  }
  // ---- mode outputs
  {
    const int nm = (int)m->mode_comp.size();
    std::vector<int4> md(std::max(nm, 1));
    std::vector<int2> fc;
    for (int v = 0; v < nm; v++) {
      if (m->mode_comp[v] < 1 || m->mode_comp[v] > 6) return fail(TLM_E_BADARG, "mode output %d: component is not Ex..Hz", v + 1);
      md[v] = int4{m->mode_ptr[v], m->mode_ptr[v + 1] - m->mode_ptr[v], m->mode_comp[v], 0};
      for (int k = m->mode_ptr[v]; k < m->mode_ptr[v + 1]; k++) {
        const int fo = m->mode_fout[k], code = m->mode_fcode[k];
        if (fo < 1 || fo > m->n_out_faces) return fail(TLM_E_BADARG, "mode output %d: face output number out of range", v + 1);
        if (code < 1 || code > 6) return fail(TLM_E_BADARG, "mode output %d: face code out of range", v + 1);
        fc.push_back(int2{fo - 1, code});
      }
    }
    std::vector<double> w = m->mode_w;
    if (fc.empty()) { fc.resize(1); w.assign(1, 0.0); }
    if ((rc = upload(m, m->mode_d, md)) || (rc = upload(m, m->mode_face, fc)) || (rc = upload(m, m->mode_wd, w))) return rc;
    if ((rc = dalloc(m, m->mode_hist, (size_t)std::max(nm, 1) * nsteps * sizeof(double)))) return rc;
    CK(cudaMemset(m->mode_hist.p, 0, m->mode_hist.bytes));
  }
  // ---- SAR volumes
  {
    const int nv = (int)m->sar_freq.size();
    std::vector<int2> ent;
    for (int v = 0; v < nv; v++)
      for (int k = m->sar_ptr[v]; k < m->sar_ptr[v + 1]; k++) {
        const int o = m->sar_out[k];
        if (o < 1 || o > m->n_out_cells) return fail(TLM_E_BADARG, "SAR volume %d: output cell %d out of range", v + 1, o);
        ent.push_back(int2{v, o - 1});
      }
    m->sar_entries = (int)ent.size();
    if (ent.empty()) ent.resize(1);
    std::vector<double2> ph((size_t)std::max(nv, 1) * nsteps, double2{0, 0});
    const double pi = 3.141592653589793;
    for (int t = 0; t < nsteps; t++) {
      const double time = (double)t * D.dt;  // (timestep-1)*dt, the time of the cell outputs
      for (int v = 0; v < nv; v++) {
        const double arg = -2.0 * pi * m->sar_freq[v] * time;
        ph[(size_t)t * nv + v] = double2{cos(arg), sin(arg)};
      }
    }
    if ((rc = upload(m, m->sar_entry, ent)) || (rc = upload(m, m->sar_phasor, ph))) return rc;
    if ((rc = dalloc(m, m->sar_acc, ent.size() * 3 * sizeof(double2)))) return rc;
    CK(cudaMemset(m->sar_acc.p, 0, m->sar_acc.bytes));
  }
  // ---- time-domain output volumes
  {
    const int nv = (int)m->ovol_gate.size() / 5;
    std::vector<tlm::OVolDev> vd(std::max(nv, 1));
    std::vector<int> cells;
    size_t off = 0;
    for (int v = 0; v < nv; v++) {
      const int *g = &m->ovol_gate[(size_t)v * 5];
      if (g[3] < 1 || g[3] > 6) return fail(TLM_E_BADARG, "output volume %d: component %d is not Ex..Hz", v + 1, g[3]);
      if (g[0] < 1 || g[2] < 1) return fail(TLM_E_BADARG, "output volume %d: first step and interval must be >= 1", v + 1);
      if (g[4] < 0 || g[4] > 2) return fail(TLM_E_BADARG, "output volume %d: kind %d is not 0, 1 or 2", v + 1, g[4]);
      const int nc = m->ovol_ptr[v + 1] - m->ovol_ptr[v];
      vd[v] = tlm::OVolDev{int4{g[0], g[1], g[2], g[3]}, g[4], nc, (int)cells.size(), (long long)off};
      for (int k = m->ovol_ptr[v]; k < m->ovol_ptr[v + 1]; k++) {
        const int o = m->ovol_out[k];
        if (o < 1 || o > m->n_out_cells) return fail(TLM_E_BADARG, "output volume %d: output cell %d out of range", v + 1, o);
        cells.push_back(o - 1);
      }
      off += (size_t)osurf_steps(g[0], g[1], g[2], nsteps) * (size_t)(g[4] == 0 ? nc : 1);
    }
    m->ovol_hist_len = off;
    if (cells.empty()) cells.resize(1);
    if ((rc = upload(m, m->ovol_dev, vd)) || (rc = upload(m, m->ovol_cells, cells))) return rc;
    if ((rc = dalloc(m, m->ovol_hist, std::max<size_t>(off, 1) * sizeof(double)))) return rc;
    CK(cudaMemset(m->ovol_hist.p, 0, m->ovol_hist.bytes));
  }
  // ---- RCS surface: faces sorted by K.x (then list order), time*c0 per step
  if (m->rcs_on) {
    const int nf = (int)m->rcs_fout.size();
    std::vector<int> order(nf);
    for (int i = 0; i < nf; i++) {
      order[i] = i;
      if (m->rcs_fout[i] < 1 || m->rcs_fout[i] > m->n_out_faces) return fail(TLM_E_BADARG, "RCS face output number out of range");
      if (m->rcs_fcode[i] < 1 || m->rcs_fcode[i] > 6) return fail(TLM_E_BADARG, "RCS face code out of range");
    }
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return m->rcs_dist[a] < m->rcs_dist[b]; });
    std::vector<int2> fc(std::max(nf, 1));
    std::vector<double> ds(std::max(nf, 1));
    for (int k = 0; k < nf; k++) {
      fc[k] = int2{m->rcs_fout[order[k]] - 1, m->rcs_fcode[order[k]]};
      ds[k] = m->rcs_dist[order[k]];
    }
    std::vector<double> tc0(nsteps);
    const double c0 = 2.99792458e8;  // CONSTANTS/constants.F90
    for (int t = 0; t < nsteps; t++) {
      double time = (double)t * D.dt;  // (timestep-1)*dt, then the half step of the face outputs
      time = time + D.dt / 2.0;
      tc0[t] = time * c0;
    }
    if ((rc = upload(m, m->rcs_face, fc)) || (rc = upload(m, m->rcs_dist_d, ds)) || (rc = upload(m, m->rcs_tc0, tc0)))
      return rc;
    if ((rc = dalloc(m, m->rcs_acc, (size_t)std::max(m->rcs_points, 1) * 4 * sizeof(double)))) return rc;
    CK(cudaMemset(m->rcs_acc.p, 0, m->rcs_acc.bytes));
  }
  if ((rc = dalloc(m, m->d_base, sizeof(int)))) return rc;
  if ((rc = dalloc(m, m->d_err, sizeof(int)))) return rc;
  CK(cudaMemset(m->d_err.p, 0, sizeof(int)));
  {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&m->n_sms, cudaDevAttrMultiProcessorCount, dev));
  }
  {
    int one = 1;
    CK(cudaMemcpy(m->d_base.p, &one, sizeof(int), cudaMemcpyHostToDevice));
  }
  if (!m->stream) {
    CK(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
    m->own_stream = true;
  }
  CK(cudaEventCreate(&m->ev0));
  CK(cudaEventCreate(&m->ev1));
  if (const char *pf = getenv("TLM_PML_PREFETCH_BLOCKS")) m->pml_prefetch = atoi(pf);
  m->side_on = side_stream_enabled((long long)m->desc.nx * m->desc.ny * m->desc.nz, false);
  if (m->side_on) {
    int rc = m->side.init();
    if (rc) return rc;
  }
  m->finalized = true;
  return TLM_OK;
}

// TMA-staged bulk kernel configurations (the autotuner's search space):
// tile elements per work item and shared-memory ring depth.
struct Variant {
  int tile32, stages32, tile64, stages64;
};
constexpr Variant kVariants[] = {
    {0, 0, 0, 0},        // 0: register-pipelined kernel (no TMA)
    {1024, 2, 512, 2},   // 1
    {512, 3, 256, 3},    // 2
    {512, 4, 256, 4},    // 3
    {1024, 3, 512, 3},   // 4
    {256, 6, 128, 6},    // 5
};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

// Tiles of TILE elements of each plane interior that hold at least one
// free-space cell.
int build_tiles(Mesh *m, int TILE) {
  if (m->tiles_tile == TILE) return TLM_OK;
  const int nx = m->desc.nx, ny = m->desc.ny, nz = m->desc.nz;
  const int per_plane = ny * m->Px;
  const int segs_pp = (per_plane + 31) / 32;
  std::vector<int4> tl;
  for (int z = 0; z < nz; z++) {
    for (int e0 = 0; e0 < per_plane; e0 += TILE) {
      const int len = std::min(TILE, per_plane - e0);
      bool any = false;
      for (int e = e0; e < e0 + len && !any; e += 32) {
        const uint32_t mk = m->host_mask[(size_t)z * segs_pp + (e >> 5)];
        for (int k = 0; k < 32 && e + k < e0 + len; k++) {
          const int x = (e + k) % m->Px;
          if (x < nx && !((mk >> k) & 1u)) {
            any = true;
            break;
          }
        }
      }
      if (any) tl.push_back(int4{z, e0, len, 0});
    }
  }
  m->n_tiles = (int)tl.size();
  m->host_tiles = tl;
  if (tl.empty()) tl.resize(1);
  int rc = upload(m, m->tiles, tl);
  if (rc) return rc;
  m->tiles_tile = TILE;
  return TLM_OK;
}

template <typename T, int VEC, int TILE, int NSTAGE>
int launch_tma(Mesh *m, const tlm::MeshDev<T> &md, int k) {
  using Cfg = tlm::TmaCfg<T, VEC, TILE, NSTAGE>;
  auto kern = tlm::tlm_bulk_tma_kernel<T, VEC, TILE, NSTAGE>;
  // the shared-memory opt-in is per device; the occupancy query is cached per device too
  static int per_sm_cache[64] = {0};
  int dev = 0;
  CK(cudaGetDevice(&dev));
  int per_sm = dev < 64 ? per_sm_cache[dev] : 0;
  if (per_sm == 0) {
    CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::SMEM));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, Cfg::THREADS, Cfg::SMEM));
    if (per_sm < 1) per_sm = 1;
    if (dev < 64) per_sm_cache[dev] = per_sm;
  }
  const int grid = std::max(1, std::min(m->n_tiles, per_sm * m->n_sms));
  tlm::TileList tl{(const int4 *)m->tiles.p, m->n_tiles, (int *)m->d_err.p};
  if (m->dry_launch) return TLM_OK;  // configuration only (outside stream capture)
  if (m->n_tiles) kern<<<grid, Cfg::THREADS, Cfg::SMEM, m->stream>>>(md, nullptr, tl, k);
  return TLM_OK;
}

// Everything a bulk launch needs that must not happen inside stream
// capture (allocation of the tile list, kernel attributes).
template <typename T, int VEC>
int launch_bulk(Mesh *m, const tlm::MeshDev<T> &md, int k);

int prepare_variant(Mesh *m) {
  if (m->variant == 0) return TLM_OK;
  const Variant &cf = kVariants[m->variant];
  int rc = build_tiles(m, m->fp64 ? cf.tile64 : cf.tile32);
  if (rc) return rc;
  m->dry_launch = true;
  rc = m->fp64 ? launch_bulk<double, 2>(m, mesh_dev<double>(m), 0) : launch_bulk<float, 4>(m, mesh_dev<float>(m), 0);
  m->dry_launch = false;
  return rc;
}

template <typename T, int VEC>
int launch_bulk(Mesh *m, const tlm::MeshDev<T> &md, int k) {
  const int v = m->variant;
  if (v == 0) {
    const int threads = 256;
    dim3 grid((md.chunks_per_plane + threads - 1) / threads, m->desc.nz);
    tlm::tlm_cell_kernel<T, VEC><<<grid, threads, 0, m->stream>>>(md, k);
    return TLM_OK;
  }
  const Variant &cf = kVariants[v];
  const int TILE = sizeof(T) == 4 ? cf.tile32 : cf.tile64;
  if (m->tiles_tile != TILE) return fail(TLM_E_STATE, "tile list not prepared for variant %d", v);
  if constexpr (sizeof(T) == 4) {
    switch (v) {
      case 1: return launch_tma<T, VEC, 1024, 2>(m, md, k);
      case 2: return launch_tma<T, VEC, 512, 3>(m, md, k);
      case 3: return launch_tma<T, VEC, 512, 4>(m, md, k);
      case 4: return launch_tma<T, VEC, 1024, 3>(m, md, k);
      default: return launch_tma<T, VEC, 256, 6>(m, md, k);
    }
  } else {
    switch (v) {
      case 1: return launch_tma<T, VEC, 512, 2>(m, md, k);
      case 2: return launch_tma<T, VEC, 256, 3>(m, md, k);
      case 3: return launch_tma<T, VEC, 256, 4>(m, md, k);
      case 4: return launch_tma<T, VEC, 512, 3>(m, md, k);
      default: return launch_tma<T, VEC, 128, 6>(m, md, k);
    }
  }
}

// Enqueue relative steps [0, n) of one step bundle (kernels only, the base
// counter is advanced by the caller).
// Compile-time bound on the Z-filter orders of a mesh's special-cell kernel
// (1, 2, 4 or the library maximum): the smallest that covers every material.
int special_order_bound(int maxo) {
  return maxo <= 1 ? 1 : (maxo <= 2 ? 2 : (maxo <= 3 ? 3 : (maxo <= 4 ? 4 : tlm::kMaxOrder)));
}

template <typename T>
void launch_special(int bound, int blocks, cudaStream_t st, const tlm::MeshDev<T> &md, int n, int k) {
  switch (bound) {
    case 1: tlm::tlm_special_kernel<T, 1><<<blocks, 128, 0, st>>>(md, n, k); break;
    case 2: tlm::tlm_special_kernel<T, 2><<<blocks, 128, 0, st>>>(md, n, k); break;
    case 3: tlm::tlm_special_kernel<T, 3><<<blocks, 128, 0, st>>>(md, n, k); break;
    case 4: tlm::tlm_special_kernel<T, 4><<<blocks, 128, 0, st>>>(md, n, k); break;
    default: tlm::tlm_special_kernel<T, tlm::kMaxOrder><<<blocks, 128, 0, st>>>(md, n, k); break;
  }
}

tlm::PmmList pmm_list(Mesh *m) {
  return tlm::PmmList{(const int4 *)m->pmm_pos.p, (const int2 *)m->pmm_parmat.p, (double *)m->pmm_state.p,
                      (const double *)m->pmm_sigma.p, m->n_pmm};
}

template <typename T, int VEC>
int enqueue_steps(Mesh *m, int n, cudaEvent_t *kev) {
  const tlm::MeshDev<T> md = mesh_dev<T>(m);
  const tlm::FaceDev fd = face_dev(m);
  const tlm::DftDev dd = dft_dev(m);
  for (int k = 0; k < n; k++) {
    if (m->small_every > 0) {
      tlm::tlm_flush_small_kernel<T><<<4 * m->n_sms, 256, 0, m->stream>>>(md, k, m->small_every, m->small_value);
      m->last_launches++;
    }
    // timed runs keep one stream, so the events around the bulk kernel time it alone
    const bool side = m->side_on && !kev && (m->n_pml_list || m->n_pmm || m->n_sp_dev);
    int rc;
    if (side && (rc = m->side.begin(m->stream))) return rc;
    if (kev) cudaEventRecord(kev[2 * k], m->stream);
    rc = launch_bulk<T, VEC>(m, md, k);
    if (rc) return rc;
    if (kev) cudaEventRecord(kev[2 * k + 1], m->stream);
    m->last_launches++;
    const cudaStream_t ss = side ? m->side.s : m->stream;
    if (m->n_pml_list) {
      tlm::PmlList pl{(const unsigned long long *)m->pml_pos.p, (const uint16_t *)m->pml_par16.p,
                      (const int2 *)m->pml_outmap.p, m->n_pml_list, m->n_pml_out, m->pml_shell,
                      m->pml_by_class ? (const double *)m->pml_cls_par.p : nullptr};
      tlm::tlm_pml_kernel<T><<<(m->n_pml_list + 127) / 128, 128, 0, ss>>>(md, pl, k, m->pml_prefetch);
      m->last_launches++;
    }
    if (m->n_pmm) {
      tlm::tlm_pml_material_kernel<T><<<(m->n_pmm + 127) / 128, 128, 0, ss>>>(md, pmm_list(m), k);
      m->last_launches++;
    }
    if (m->n_sp_dev) {
      launch_special<T>(special_order_bound(std::max(m->filt_eo, m->filt_mo)), (m->n_sp_dev + 127) / 128, ss, md,
                        m->n_sp_dev, k);
      m->last_launches++;
    }
    if (side && (rc = m->side.end(m->stream))) return rc;
    if (m->vdft_entries) {  // reads the cell outputs this step's cell kernels wrote
      const tlm::VolDftDev vd = vol_dft_dev(m);
      tlm::tlm_volume_dft_kernel<<<(vd.n_entries + 255) / 256, 256, 0, m->stream>>>(vd, md.d_base, k);
      m->last_launches++;
    }
    if (m->sar_entries) {  // likewise
      const tlm::SarDev sd = sar_dev(m);
      tlm::tlm_sar_kernel<<<(sd.n_entries + 255) / 256, 256, 0, m->stream>>>(sd, md.d_base, k);
      m->last_launches++;
    }
    if (!m->ovol_gate.empty()) {  // likewise
      const tlm::OutVolDev ov = out_vol_dev(m);
      tlm::tlm_output_volume_kernel<<<ov.n_vol, tlm::kOutVolThreads, 0, m->stream>>>(ov, md.d_base, k);
      m->last_launches++;
    }
    if (fd.n_faces) {
      tlm::tlm_face_kernel<T><<<(fd.n_faces + 127) / 128, 128, 0, m->stream>>>(md, fd, k);
      m->last_launches++;
    }
    if (!m->fpr_face.empty()) {
      const tlm::FaceProbeDev pd = face_probe_dev(m);
      tlm::tlm_face_probe_kernel<<<(pd.n + 127) / 128, 128, 0, m->stream>>>(pd, fd.face_field, md.d_base, k);
      m->last_launches++;
    }
    if (m->osurf_entries) {  // reads the face fields the face kernel wrote
      const tlm::OutSurfDev od = out_surf_dev(m);
      tlm::tlm_output_surface_kernel<<<(od.n_entries + 255) / 256, 256, 0, m->stream>>>(od, md.d_base, k);
      m->last_launches++;
    }
    if (m->rcs_on && !m->rcs_fout.empty()) {
      const tlm::RcsDev rd = rcs_dev(m);
      tlm::tlm_rcs_kernel<<<(rd.n_faces + 255) / 256, 256, 0, m->stream>>>(rd, md.d_base, k);
      m->last_launches++;
    }
    if (m->ps_entries) {
      const tlm::PowerSurfDev pd2 = power_surf_dev(m);
      tlm::tlm_power_surface_kernel<<<(pd2.n_entries + 255) / 256, 256, 0, m->stream>>>(pd2, md.d_base, k);
      m->last_launches++;
    }
    if (!m->mode_comp.empty()) {
      const tlm::ModeDev mdv = mode_dev(m);
      tlm::tlm_mode_kernel<<<mdv.n_modes, tlm::kOutVolThreads, 0, m->stream>>>(mdv, md.d_base, k);
      m->last_launches++;
    }
    if (m->hs_outer && m->hs_n) {
      tlm::tlm_outer_huygens_kernel<T><<<(m->hs_n + 127) / 128, 128, 0, m->stream>>>(md, outer_hs_dev(m), k);
      m->last_launches++;
    }
    if (m->ff_entries) {
      const tlm::FarFieldDev fdv = far_field_dev(m);
      tlm::tlm_far_field_kernel<<<(fdv.n_entries + 255) / 256, 256, 0, m->stream>>>(fdv, md.d_base, k);
      m->last_launches++;
    }
    if (dd.n_entries) {
      tlm::tlm_dft_kernel<<<(dd.n_entries + 255) / 256, 256, 0, m->stream>>>(dd, md.d_base, k);
      m->last_launches++;
    }
  }
  CK(cudaGetLastError());
  return TLM_OK;
}

int enqueue(Mesh *m, int n, cudaEvent_t *kev) {
  return m->fp64 ? enqueue_steps<double, 2>(m, n, kev) : enqueue_steps<float, 4>(m, n, kev);
}

int run_steps(Mesh *m, int n) {
  int rc;
  if ((rc = prepare_variant(m))) return rc;
  m->last_launches = 0;
  CK(cudaEventRecord(m->ev0, m->stream));
  if (m->timing) {
    // per-step launches with an event pair around every cell kernel; the
    // durations are summed once the run has finished (last_run_time)
    const size_t need = 2 * (size_t)n;
    while (m->kev.size() < need) {
      cudaEvent_t e;
      CK(cudaEventCreate(&e));
      m->kev.push_back(e);
    }
    for (int s = 0; s < n; s++) {
      if ((rc = enqueue(m, 1, m->kev.data() + 2 * s))) return rc;
      tlm::tlm_advance_base<<<1, 1, 0, m->stream>>>((int *)m->d_base.p, 1);
      m->last_launches++;
    }
    m->timed_steps = n;
  } else {
    const int G = Mesh::kGraphSteps;
    int full = n / G, rem = n % G;
    if (full > 0 && !m->graph) {
      cudaGraph_t g;
      CK(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
      long long saved = m->last_launches;
      rc = enqueue(m, G, nullptr);
      tlm::tlm_advance_base<<<1, 1, 0, m->stream>>>((int *)m->d_base.p, G);
      cudaError_t ce = cudaStreamEndCapture(m->stream, &g);
      if (rc) return rc;
      if (ce != cudaSuccess) return fail(TLM_E_CUDA, "graph capture: %s", cudaGetErrorString(ce));
      ce = cudaGraphInstantiate(&m->graph, g, 0);
      cudaGraphDestroy(g);
      if (ce != cudaSuccess) return fail(TLM_E_CUDA, "graph instantiate: %s", cudaGetErrorString(ce));
      m->graph_launches = m->last_launches - saved + 1;  // the kernels captured, + the counter advance
      m->last_launches = saved;
    }
    for (int i = 0; i < full; i++) {
      CK(cudaGraphLaunch(m->graph, m->stream));
      m->last_launches += m->graph_launches;
    }
    for (int i = 0; i < rem; i++) {
      if ((rc = enqueue(m, 1, nullptr))) return rc;
      tlm::tlm_advance_base<<<1, 1, 0, m->stream>>>((int *)m->d_base.p, 1);
      m->last_launches++;
    }
    m->timed_steps = 0;
  }
  CK(cudaEventRecord(m->ev1, m->stream));
  CK(cudaGetLastError());
  return TLM_OK;
}

}  // namespace

extern "C" {

int tlm_gpu_create(const tlm_gpu_mesh_desc *desc, int64_t *handle) {
  if (!desc || !handle) return fail(TLM_E_BADARG, "null argument");
  if (desc->nx < 1 || desc->ny < 1 || desc->nz < 1) return fail(TLM_E_BADARG, "mesh dimensions must be >= 1");
  if (desc->n_timesteps < 1) return fail(TLM_E_BADARG, "n_timesteps must be >= 1");
  if (!(desc->dl > 0) || !(desc->dt > 0)) return fail(TLM_E_BADARG, "dl and dt must be positive");
  if (desc->precision != TLM_PRECISION_FP32 && desc->precision != TLM_PRECISION_FP64)
    return fail(TLM_E_BADARG, "precision must be TLM_PRECISION_FP32 or TLM_PRECISION_FP64");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(TLM_E_CUDA, "no CUDA device available");
  if (desc->device < 0 || desc->device >= ndev) return fail(TLM_E_BADARG, "device %d out of range", desc->device);
  auto m = std::make_unique<Mesh>();
  m->desc = *desc;
  m->fp64 = desc->precision == TLM_PRECISION_FP64;
  m->Px = ((desc->nx + 1 + 3) / 4) * 4;
  m->Py = desc->ny + 2;
  m->Pz = desc->nz + 2;
  m->plane = (long long)m->Px * m->Py * m->Pz;
  if ((long long)desc->ny * m->Px >= (1LL << 31) / 4) return fail(TLM_E_BADARG, "mesh plane too large");
  std::lock_guard<std::mutex> lk(g_mu);
  const int64_t h = g_next++;
  g_meshes[h] = std::move(m);
  *handle = h;
  return TLM_OK;
}

int tlm_gpu_set_cells(int64_t h, const int32_t *code, int32_t n_special, const int32_t *sp_material,
                      const int32_t *sp_pml, const int32_t *sp_excitation, const int32_t *sp_output) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->finalized) return fail(TLM_E_STATE, "tables are fixed after the first run");
  if (!code || n_special < 0 || (n_special && (!sp_material || !sp_pml || !sp_excitation || !sp_output)))
    return fail(TLM_E_BADARG, "null argument");
  const long long ncell = (long long)m->desc.nx * m->desc.ny * m->desc.nz;
  m->cell_code.assign(code, code + ncell);
  m->n_special = n_special;
  m->sp_material.assign(sp_material, sp_material + n_special);
  m->sp_pml.assign(sp_pml, sp_pml + n_special);
  m->sp_exc.assign(sp_excitation, sp_excitation + n_special);
  m->sp_out.assign(sp_output, sp_output + n_special);
  m->have_cells = true;
  return TLM_OK;
}

int tlm_gpu_set_materials(int64_t h, int32_t n, const int32_t *type, const int32_t *eps_exists, const int32_t *mu_exists,
                          const int32_t *eps_order, const int32_t *mu_order, const double *Ys_eps_f,
                          const double *Zs_mu_f, const double *Ge, const double *Rm, const double *eps_a,
                          const double *eps_b, const double *mu_a, const double *mu_b, int32_t stride) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->finalized) return fail(TLM_E_STATE, "tables are fixed after the first run");
  if (n < 0) return fail(TLM_E_BADARG, "negative material count");
  m->mats.assign(n, tlm::MatDev{});
  for (int i = 0; i < n; i++) {
    tlm::MatDev &d = m->mats[i];
    d.type = type[i];
    if (d.type < 1 || d.type > 3) return fail(TLM_E_UNSUPPORTED, "volume material %d: type %d not supported", i + 1, d.type);
    d.eps_exists = eps_exists[i];
    d.mu_exists = mu_exists[i];
    d.eps_order = eps_order[i];
    d.mu_order = mu_order[i];
    if (d.eps_order < 0 || d.eps_order > tlm::kMaxOrder || d.mu_order < 0 || d.mu_order > tlm::kMaxOrder ||
        d.eps_order + 1 > stride || d.mu_order + 1 > stride)
      return fail(TLM_E_UNSUPPORTED, "volume material %d: filter order above %d", i + 1, tlm::kMaxOrder);
    d.Ys_eps_f = Ys_eps_f[i];
    d.Zs_mu_f = Zs_mu_f[i];
    d.Ge = Ge[i];
    d.Rm = Rm[i];
    for (int k = 0; k <= tlm::kMaxOrder; k++) {
      d.eps_a[k] = k <= d.eps_order ? eps_a[(size_t)i * stride + k] : 0.0;
      d.eps_b[k] = k <= d.eps_order ? eps_b[(size_t)i * stride + k] : 0.0;
      d.mu_a[k] = k <= d.mu_order ? mu_a[(size_t)i * stride + k] : 0.0;
      d.mu_b[k] = k <= d.mu_order ? mu_b[(size_t)i * stride + k] : 0.0;
    }
    if (d.type == 3 && ((d.eps_exists && d.eps_b[0] == 0.0) || (d.mu_exists && d.mu_b[0] == 0.0)))
      return fail(TLM_E_BADARG, "volume material %d: filter b(0) is zero", i + 1);
    // reciprocals of the constant divisors of special_cell, each divisor
    // formed exactly as the cell update forms it
    {
      const double Y04 = tlm::kY0 * 4.0, Z04 = tlm::kZ0 * 4.0;
      d.inv_eps_b0 = d.eps_b[0] != 0.0 ? 1.0 / d.eps_b[0] : 0.0;
      d.inv_mu_b0 = d.mu_b[0] != 0.0 ? 1.0 / d.mu_b[0] : 0.0;
      double Y = Y04;
      d.inv_Y_eps = 1.0 / (Y + (d.eps_exists ? d.Ys_eps_f : 0.0));
      if (d.eps_exists) Y = Y + d.Ys_eps_f;
      d.inv_Y_Ge = 1.0 / (Y + d.Ge);
      double Z = Z04;
      if (d.mu_exists) Z = Z + d.Zs_mu_f;
      Z = Z + d.Rm;
      d.inv_Z = 1.0 / Z;
    }
  }
  return TLM_OK;
}

int tlm_gpu_set_pml(int64_t h, int32_t n_params, const double *params, int32_t n_pml_cells, const int32_t *cell_param) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->finalized) return fail(TLM_E_STATE, "tables are fixed after the first run");
  if (n_params < 0 || n_pml_cells < 0 || (n_params && !params) || (n_pml_cells && !cell_param))
    return fail(TLM_E_BADARG, "bad PML arguments");
  m->n_pml_params = n_params;
  m->pml_params.assign(params, params + (size_t)n_params * 15);
  m->n_pml_cells = n_pml_cells;
  m->pml_cell_param.assign(cell_param, cell_param + n_pml_cells);
  return TLM_OK;
}

int tlm_gpu_set_pml_sigma(int64_t h, int32_t n_params, const double *sigma) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->finalized) return fail(TLM_E_STATE, "tables are fixed after the first run");
  if (n_params != m->n_pml_params || (n_params && !sigma))
    return fail(TLM_E_BADARG, "PML sigma rows: %d given, %d PML parameter rows set", n_params, m->n_pml_params);
  m->pml_sigma.assign(sigma, sigma + (size_t)n_params * 3);
  return TLM_OK;
}

int tlm_gpu_set_excitation(int64_t h, int32_t n_fn, int32_t n_steps, const double *value, const double *value_face,
                           int32_t n_points, const int32_t *pt_cell, const int32_t *pt_comp, const int32_t *pt_fn,
                           const int32_t *pt_type, int32_t n_exc_cells) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->finalized) return fail(TLM_E_STATE, "tables are fixed after the first run");
  if (n_fn < 0 || n_steps < 0 || n_points < 0 || n_exc_cells < 0) return fail(TLM_E_BADARG, "negative count");
  m->n_fn = n_fn;
  m->n_fn_steps = n_steps;
  m->fn_value.assign(value, value + (size_t)n_fn * n_steps);
  m->fn_value_face.assign(value_face, value_face + (size_t)n_fn * n_steps);
  m->pt_cell.assign(pt_cell, pt_cell + n_points);
  m->pt_comp.assign(pt_comp, pt_comp + n_points);
  m->pt_fn.assign(pt_fn, pt_fn + n_points);
  m->pt_type.assign(pt_type, pt_type + n_points);
  for (int i = 0; i < n_points; i++)
    if (pt_type[i] != 0 && pt_type[i] != 1) return fail(TLM_E_BADARG, "point excitation %d: bad source type", i + 1);
  m->n_exc_cells = n_exc_cells;
  return TLM_OK;
}

int tlm_gpu_set_faces(int64_t h, int32_t n, const int32_t *cx, const int32_t *cy, const int32_t *cz, const int32_t *dir,
                      const int32_t *exc, const int32_t *out, int32_t n_exc_faces, int32_t n_out_faces) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->finalized) return fail(TLM_E_STATE, "tables are fixed after the first run");
  if (n < 0) return fail(TLM_E_BADARG, "negative face count");
  m->f_cx.assign(cx, cx + n);
  m->f_cy.assign(cy, cy + n);
  m->f_cz.assign(cz, cz + n);
  m->f_dir.assign(dir, dir + n);
  m->f_exc.assign(exc, exc + n);
  m->f_out.assign(out, out + n);
  m->n_exc_faces = n_exc_faces;
  m->n_out_faces = n_out_faces;
  return TLM_OK;
}

int tlm_gpu_set_face_materials(int64_t h, int32_t n, const int32_t *type) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->finalized) return fail(TLM_E_STATE, "tables are fixed after the first run");
  if (n < 0 || (n && !type)) return fail(TLM_E_BADARG, "bad face material arguments");
  m->f_mat.assign(type, type + n);
  return TLM_OK;
}

int tlm_gpu_set_thin_layers(int64_t h, int32_t n, const double *f, const double *a, const double *b,
                            const int32_t *order, int32_t stride) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->finalized) return fail(TLM_E_STATE, "tables are fixed after the first run");
  if (n < 0 || (n && (!f || !a || !b || !order)) || stride < 1)
    return fail(TLM_E_BADARG, "bad thin-layer arguments");
  m->thin.assign(n, tlm::ThinLayerDev{});
  for (int i = 0; i < n; i++)
    for (int p = 0; p < 3; p++)
      for (int k = 0; k < 4; k++) {
        const size_t e = ((size_t)i * 3 + p) * 4 + k;
        const int o = order[e];
        if (o < 0 || o > tlm::kMaxOrder || o + 1 > stride)
          return fail(TLM_E_UNSUPPORTED, "thin layer %d: filter order %d (at most %d)", i + 1, o, tlm::kMaxOrder);
        tlm::ThinLayerDev &d = m->thin[i];
        d.order[p][k] = o;
        d.f[p][k] = f[e];
        for (int c = 0; c <= tlm::kMaxOrder; c++) {
          d.a[p][k][c] = c <= o ? a[e * stride + c] : 0.0;
          d.b[p][k][c] = c <= o ? b[e * stride + c] : 0.0;
        }
        if (d.b[p][k][0] == 0.0) return fail(TLM_E_BADARG, "thin layer %d: filter b(0) is zero", i + 1);
      }
  for (int i = 0; i < n; i++)  // surface_material_update stops on a singular impedance matrix
    for (int p = 0; p < 3; p++)
      for (int rev = 0; rev < 2; rev++) {
        const tlm::ThinLayerDev &d = m->thin[i];
        const double U11 = tlm::kZ0 + d.f[p][0], U22 = tlm::kZ0 + d.f[p][3];
        if (U11 * U22 - d.f[p][2] * d.f[p][1] == 0.0)
          return fail(TLM_E_BADARG, "thin layer %d: singular impedance matrix", i + 1);
      }
  return TLM_OK;
}

int tlm_gpu_set_wrap(int64_t h, int32_t wrap_x, int32_t wrap_y, int32_t wrap_z) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->finalized) return fail(TLM_E_STATE, "tables are fixed after the first run");
  for (int v : {wrap_x, wrap_y, wrap_z})
    if (v != 0 && v != 1) return fail(TLM_E_BADARG, "wrapping flags must be 0 or 1");
  m->wrap = wrap_x | (wrap_y << 1) | (wrap_z << 2);
  return TLM_OK;
}

int tlm_gpu_set_face_thin_layers(int64_t h, int32_t n, const int32_t *material) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->finalized) return fail(TLM_E_STATE, "tables are fixed after the first run");
  if (n < 0 || (n && !material)) return fail(TLM_E_BADARG, "bad face thin-layer arguments");
  m->f_smat.assign(material, material + n);
  return TLM_OK;
}

int tlm_gpu_set_face_excitation(int64_t h, int32_t n, const int32_t *face_exc, const int32_t *comp,
                                const int32_t *function, const int32_t *type) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->finalized) return fail(TLM_E_STATE, "tables are fixed after the first run");
  if (n < 0 || (n && (!face_exc || !comp || !function || !type))) return fail(TLM_E_BADARG, "bad face excitation arguments");
  m->fpt_face.assign(face_exc, face_exc + n);
  m->fpt_comp.assign(comp, comp + n);
  m->fpt_fn.assign(function, function + n);
  m->fpt_type.assign(type, type + n);
  return TLM_OK;
}

int tlm_gpu_set_face_excitation_side(int64_t h, int32_t n, const int32_t *side) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->finalized) return fail(TLM_E_STATE, "tables are fixed after the first run");
  if (n < 0 || (n && !side)) return fail(TLM_E_BADARG, "bad face excitation side arguments");
  m->fpt_side.assign(side, side + n);
  return TLM_OK;
}

int tlm_gpu_set_face_excitation_scale(int64_t h, int32_t n, const double *scale) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->finalized) return fail(TLM_E_STATE, "tables are fixed after the first run");
  if (n < 0 || (n && !scale)) return fail(TLM_E_BADARG, "bad face excitation scale arguments");
  for (int e = 0; e < n; e++)
    if (!std::isfinite(scale[e])) return fail(TLM_E_BADARG, "face source %d: scale is not finite", e + 1);
  m->fpt_scale.assign(scale, scale + n);
  return TLM_OK;
}

int tlm_gpu_set_face_outputs(int64_t h, int32_t n, const int32_t *face_out, const int32_t *side, const int32_t *comp) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->finalized) return fail(TLM_E_STATE, "tables are fixed after the first run");
  if (n < 0 || (n && (!face_out || !side || !comp))) return fail(TLM_E_BADARG, "bad face output arguments");
  m->fpr_face.assign(face_out, face_out + n);
  m->fpr_side.assign(side, side + n);
  m->fpr_comp.assign(comp, comp + n);
  return TLM_OK;
}

int tlm_gpu_set_huygens(int64_t h, int32_t n, const int32_t *face_exc, const int32_t *norm, const double *offset,
                        const double *Ei, const double *Hi, double offset_min, double c, int32_t function) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->finalized) return fail(TLM_E_STATE, "tables are fixed after the first run");
  if (n < 0 || (n && (!face_exc || !norm || !offset || !Ei || !Hi))) return fail(TLM_E_BADARG, "bad Huygens arguments");
  m->hs_n = n;
  m->hs_face_exc.assign(face_exc, face_exc + n);
  m->hs_norm.assign(norm, norm + 3 * (size_t)n);
  m->hs_offset.assign(offset, offset + n);
  for (int i = 0; i < 3 && n; i++) {
    m->hs_Ei[i] = Ei[i];
    m->hs_Hi[i] = Hi[i];
  }
  m->hs_offset_min = offset_min;
  m->hs_c = c;
  m->hs_fn = function;
  if (n && !(c > 0)) return fail(TLM_E_BADARG, "Huygens wave speed must be positive");
  return TLM_OK;
}

int tlm_gpu_set_outer_huygens(int64_t h, int32_t n, const int32_t *cell_face, const double *offset, const double *Ei,
                              const double *Hi, double offset_min, double c, int32_t function) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->finalized) return fail(TLM_E_STATE, "tables are fixed after the first run");
  if (n < 0 || (n && (!cell_face || !offset || !Ei || !Hi))) return fail(TLM_E_BADARG, "bad outer Huygens arguments");
  if (n && !(c > 0)) return fail(TLM_E_BADARG, "Huygens wave speed must be positive");
  m->hs_outer = n > 0;
  m->hs_n = n;
  m->hs_cell.assign(cell_face, cell_face + 4 * (size_t)n);
  m->hs_offset.assign(offset, offset + n);
  m->hs_face_exc.assign(n, 0);
  m->hs_norm.assign(3 * (size_t)n, 0);
  for (int i = 0; i < 3; i++) {
    m->hs_Ei[i] = Ei[i];
    m->hs_Hi[i] = Hi[i];
  }
  m->hs_offset_min = offset_min;
  m->hs_c = c;
  m->hs_fn = function;
  return TLM_OK;
}

int tlm_gpu_set_outputs(int64_t h, int32_t n_out_cells) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->finalized) return fail(TLM_E_STATE, "tables are fixed after the first run");
  if (n_out_cells < 0) return fail(TLM_E_BADARG, "negative output count");
  m->n_out_cells = n_out_cells;
  return TLM_OK;
}

int tlm_gpu_set_output_series(int64_t h, int32_t n, const int32_t *keep) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->finalized) return fail(TLM_E_STATE, "tables are fixed after the first run");
  if (n < 0 || (n && !keep)) return fail(TLM_E_BADARG, "bad output series flags");
  for (int i = 0; i < n; i++)
    if (keep[i] != 0 && keep[i] != 1) return fail(TLM_E_BADARG, "output series flag %d is not 0 or 1", i + 1);
  m->out_keep.assign(keep, keep + n);
  return TLM_OK;
}

int tlm_gpu_set_volume_dft(int64_t h, int32_t n, const double *freq, const int32_t *component,
                           const int32_t *first_step, const int32_t *last_step, const int32_t *interval,
                           const int32_t *ptr, const int32_t *out_cells) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->finalized) return fail(TLM_E_STATE, "tables are fixed after the first run");
  if (n < 0 || (n && (!freq || !component || !first_step || !last_step || !interval || !ptr || !out_cells)))
    return fail(TLM_E_BADARG, "bad output volume arguments");
  for (int v = 0; v < n; v++)
    if (ptr[v] < 0 || ptr[v + 1] < ptr[v]) return fail(TLM_E_BADARG, "output volume cell pointers must be non-decreasing");
  m->vdft_freq.assign(freq, freq + n);
  m->vdft_gate.resize((size_t)n * 4);
  for (int v = 0; v < n; v++) {
    m->vdft_gate[(size_t)v * 4 + 0] = first_step[v];
    m->vdft_gate[(size_t)v * 4 + 1] = last_step[v];
    m->vdft_gate[(size_t)v * 4 + 2] = interval[v];
    m->vdft_gate[(size_t)v * 4 + 3] = component[v];
  }
  m->vdft_ptr.assign(ptr, ptr + (n ? n + 1 : 0));
  const int ne = n ? ptr[n] : 0;
  m->vdft_out.assign(out_cells, out_cells + ne);
  return TLM_OK;
}

int tlm_gpu_set_output_surfaces(int64_t h, int32_t n, const int32_t *component, const int32_t *first_step,
                                const int32_t *last_step, const int32_t *interval, const int32_t *both_sides,
                                const int32_t *face_ptr, const int32_t *face_out, const int32_t *face_code) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->finalized) return fail(TLM_E_STATE, "tables are fixed after the first run");
  if (n < 0 || (n && (!component || !first_step || !last_step || !interval || !both_sides || !face_ptr ||
                      !face_out || !face_code)))
    return fail(TLM_E_BADARG, "bad output surface arguments");
  for (int v = 0; v < n; v++)
    if (face_ptr[v] < 0 || face_ptr[v + 1] < face_ptr[v])
      return fail(TLM_E_BADARG, "output surface face pointers must be non-decreasing");
  m->osurf_gate.resize((size_t)n * 5);
  for (int v = 0; v < n; v++) {
    int *g = &m->osurf_gate[(size_t)v * 5];
    g[0] = first_step[v]; g[1] = last_step[v]; g[2] = interval[v]; g[3] = component[v]; g[4] = both_sides[v];
  }
  m->osurf_ptr.assign(face_ptr, face_ptr + (n ? n + 1 : 0));
  const int ne = n ? face_ptr[n] : 0;
  m->osurf_fout.assign(face_out, face_out + ne);
  m->osurf_fcode.assign(face_code, face_code + ne);
  return TLM_OK;
}

int tlm_gpu_set_rcs(int64_t h, double theta, double phi, int32_t points_per_cell, int32_t n_points,
                    int32_t point_offset, int32_t n_faces, const int32_t *face_out, const int32_t *face_code,
                    const double *face_dist) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->finalized) return fail(TLM_E_STATE, "tables are fixed after the first run");
  if (points_per_cell < 1 || n_points < 1 || n_faces < 0 || (n_faces && (!face_out || !face_code || !face_dist)))
    return fail(TLM_E_BADARG, "bad RCS surface arguments");
  m->rcs_on = true;
  m->rcs_theta = theta;
  m->rcs_phi = phi;
  m->rcs_npc = points_per_cell;
  m->rcs_points = n_points;
  m->rcs_offset = point_offset;
  m->rcs_fout.assign(face_out, face_out + n_faces);
  m->rcs_fcode.assign(face_code, face_code + n_faces);
  m->rcs_dist.assign(face_dist, face_dist + n_faces);
  return TLM_OK;
}

int tlm_gpu_set_output_volumes(int64_t h, int32_t n, const int32_t *kind, const int32_t *component,
                               const int32_t *first_step, const int32_t *last_step, const int32_t *interval,
                               const int32_t *cell_ptr, const int32_t *cell_out) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->finalized) return fail(TLM_E_STATE, "tables are fixed after the first run");
  if (n < 0 || (n && (!kind || !component || !first_step || !last_step || !interval || !cell_ptr || !cell_out)))
    return fail(TLM_E_BADARG, "bad output volume arguments");
  for (int v = 0; v < n; v++)
    if (cell_ptr[v] < 0 || cell_ptr[v + 1] < cell_ptr[v])
      return fail(TLM_E_BADARG, "output volume cell pointers must be non-decreasing");
  m->ovol_gate.resize((size_t)n * 5);
  for (int v = 0; v < n; v++) {
    int *g = &m->ovol_gate[(size_t)v * 5];
    g[0] = first_step[v]; g[1] = last_step[v]; g[2] = interval[v]; g[3] = component[v]; g[4] = kind[v];
  }
  m->ovol_ptr.assign(cell_ptr, cell_ptr + (n ? n + 1 : 0));
  const int ne = n ? cell_ptr[n] : 0;
  m->ovol_out.assign(cell_out, cell_out + ne);
  return TLM_OK;
}

int tlm_gpu_fetch_output_volumes(int64_t h, double *out) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->batch_stream) CK(cudaStreamSynchronize(m->batch_stream));
  if (!m->finalized) return fail(TLM_E_STATE, "no run yet");
  if (!m->ovol_hist_len) return TLM_OK;
  CK(cudaStreamSynchronize(m->stream));
  CK(cudaMemcpy(out, m->ovol_hist.p, m->ovol_hist_len * sizeof(double), cudaMemcpyDeviceToHost));
  return TLM_OK;
}

int tlm_gpu_set_power_surfaces(int64_t h, int32_t n, const double *freq, const int32_t *face_ptr,
                               const int32_t *face_out, const int32_t *face_code) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->finalized) return fail(TLM_E_STATE, "tables are fixed after the first run");
  if (n < 0 || (n && (!freq || !face_ptr || !face_out || !face_code))) return fail(TLM_E_BADARG, "bad power surface arguments");
  for (int v = 0; v < n; v++)
    if (face_ptr[v] < 0 || face_ptr[v + 1] < face_ptr[v])
      return fail(TLM_E_BADARG, "power surface face pointers must be non-decreasing");
  m->ps_freq.assign(freq, freq + n);
  m->ps_ptr.assign(face_ptr, face_ptr + (n ? n + 1 : 0));
  const int ne = n ? face_ptr[n] : 0;
  m->ps_fout.assign(face_out, face_out + ne);
  m->ps_fcode.assign(face_code, face_code + ne);
  return TLM_OK;
}

int tlm_gpu_fetch_power_surfaces(int64_t h, double *out) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->batch_stream) CK(cudaStreamSynchronize(m->batch_stream));
  if (!m->finalized) return fail(TLM_E_STATE, "no run yet");
  if (!m->ps_entries) return TLM_OK;
  CK(cudaStreamSynchronize(m->stream));
  CK(cudaMemcpy(out, m->ps_acc.p, (size_t)m->ps_entries * 8 * sizeof(double), cudaMemcpyDeviceToHost));
  return TLM_OK;
}

int tlm_gpu_set_mode_outputs(int64_t h, int32_t n, const int32_t *component, const int32_t *face_ptr,
                             const int32_t *face_out, const int32_t *face_code, const double *mode_field) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->finalized) return fail(TLM_E_STATE, "tables are fixed after the first run");
  if (n < 0 || (n && (!component || !face_ptr || !face_out || !face_code || !mode_field)))
    return fail(TLM_E_BADARG, "bad mode output arguments");
  for (int v = 0; v < n; v++)
    if (face_ptr[v] < 0 || face_ptr[v + 1] < face_ptr[v])
      return fail(TLM_E_BADARG, "mode output face pointers must be non-decreasing");
  m->mode_comp.assign(component, component + n);
  m->mode_ptr.assign(face_ptr, face_ptr + (n ? n + 1 : 0));
  const int ne = n ? face_ptr[n] : 0;
  m->mode_fout.assign(face_out, face_out + ne);
  m->mode_fcode.assign(face_code, face_code + ne);
  m->mode_w.assign(mode_field, mode_field + ne);
  return TLM_OK;
}

int tlm_gpu_fetch_mode_outputs(int64_t h, int32_t first, int32_t n, double *out) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->batch_stream) CK(cudaStreamSynchronize(m->batch_stream));
  if (!m->finalized) return fail(TLM_E_STATE, "no run yet");
  if (first < 1 || n < 0 || first + n - 1 >= m->next_step) return fail(TLM_E_BADARG, "steps not yet computed");
  const size_t nm = m->mode_comp.size();
  if (!nm || !n) return TLM_OK;
  CK(cudaStreamSynchronize(m->stream));
  CK(cudaMemcpy(out, (double *)m->mode_hist.p + (size_t)(first - 1) * nm, (size_t)n * nm * sizeof(double),
                cudaMemcpyDeviceToHost));
  return TLM_OK;
}

int tlm_gpu_set_sar_volumes(int64_t h, int32_t n, const double *freq, const int32_t *cell_ptr,
                            const int32_t *cell_out) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->finalized) return fail(TLM_E_STATE, "tables are fixed after the first run");
  if (n < 0 || (n && (!freq || !cell_ptr || !cell_out))) return fail(TLM_E_BADARG, "bad SAR volume arguments");
  for (int v = 0; v < n; v++)
    if (cell_ptr[v] < 0 || cell_ptr[v + 1] < cell_ptr[v])
      return fail(TLM_E_BADARG, "SAR volume cell pointers must be non-decreasing");
  m->sar_freq.assign(freq, freq + n);
  m->sar_ptr.assign(cell_ptr, cell_ptr + (n ? n + 1 : 0));
  const int ne = n ? cell_ptr[n] : 0;
  m->sar_out.assign(cell_out, cell_out + ne);
  return TLM_OK;
}

int tlm_gpu_fetch_sar_volumes(int64_t h, double *out) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->batch_stream) CK(cudaStreamSynchronize(m->batch_stream));
  if (!m->finalized) return fail(TLM_E_STATE, "no run yet");
  if (!m->sar_entries) return TLM_OK;
  CK(cudaStreamSynchronize(m->stream));
  CK(cudaMemcpy(out, m->sar_acc.p, (size_t)m->sar_entries * 6 * sizeof(double), cudaMemcpyDeviceToHost));
  return TLM_OK;
}

int tlm_gpu_fetch_rcs(int64_t h, double *out) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->batch_stream) CK(cudaStreamSynchronize(m->batch_stream));
  if (!m->finalized) return fail(TLM_E_STATE, "no run yet");
  if (!m->rcs_on) return TLM_OK;
  CK(cudaStreamSynchronize(m->stream));
  CK(cudaMemcpy(out, m->rcs_acc.p, (size_t)m->rcs_points * 4 * sizeof(double), cudaMemcpyDeviceToHost));
  return TLM_OK;
}

int tlm_gpu_fetch_output_surfaces(int64_t h, double *out) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->batch_stream) CK(cudaStreamSynchronize(m->batch_stream));
  if (!m->finalized) return fail(TLM_E_STATE, "no run yet");
  if (!m->osurf_hist_len) return TLM_OK;
  CK(cudaStreamSynchronize(m->stream));
  CK(cudaMemcpy(out, m->osurf_hist.p, m->osurf_hist_len * sizeof(double), cudaMemcpyDeviceToHost));
  return TLM_OK;
}

int tlm_gpu_fetch_volume_dft(int64_t h, double *out) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->batch_stream) CK(cudaStreamSynchronize(m->batch_stream));
  if (!m->finalized) return fail(TLM_E_STATE, "no run yet");
  if (!m->vdft_entries) return TLM_OK;
  CK(cudaStreamSynchronize(m->stream));
  CK(cudaMemcpy(out, m->vdft_acc.p, (size_t)m->vdft_entries * 2 * sizeof(double), cudaMemcpyDeviceToHost));
  return TLM_OK;
}

int tlm_gpu_set_small_to_zero(int64_t h, int32_t n_small, double small) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->finalized) return fail(TLM_E_STATE, "tables are fixed after the first run");
  if (n_small < 0 || !(small >= 0.0)) return fail(TLM_E_BADARG, "set_small_to_zero needs n >= 0 and value >= 0");
  m->small_every = n_small;
  m->small_value = small;
  return TLM_OK;
}

int tlm_gpu_set_dft(int64_t h, int32_t n, const double *freq, const int32_t *comp, const int32_t *ptr,
                    const int32_t *fout, const int32_t *fcode) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->finalized) return fail(TLM_E_STATE, "tables are fixed after the first run");
  if (n < 0) return fail(TLM_E_BADARG, "negative surface count");
  m->n_dft = n;
  m->dft_freq.assign(freq, freq + n);
  m->dft_comp.assign(comp, comp + n);
  m->dft_ptr.assign(ptr, ptr + n + 1);
  const int ne = n ? ptr[n] : 0;
  m->dft_fout.assign(fout, fout + ne);
  m->dft_fcode.assign(fcode, fcode + ne);
  for (int k = 0; k < ne; k++)
    if (fcode[k] < 1 || fcode[k] > 6) return fail(TLM_E_BADARG, "DFT face code out of range");
  return TLM_OK;
}

int tlm_gpu_set_dft_gate(int64_t h, int32_t n, const int32_t *first, const int32_t *last,
                         const int32_t *interval) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->finalized) return fail(TLM_E_STATE, "tables are fixed after the first run");
  if (n != m->n_dft) return fail(TLM_E_BADARG, "gate count %d differs from the %d surfaces of tlm_gpu_set_dft", n, m->n_dft);
  if (n && (!first || !last || !interval)) return fail(TLM_E_BADARG, "null gate array");
  m->dft_gate.clear();
  for (int d = 0; d < n; d++) {
    if (first[d] < 1 || interval[d] < 1) return fail(TLM_E_BADARG, "DFT gate of surface %d: first and interval >= 1", d);
    m->dft_gate.push_back(first[d]);
    m->dft_gate.push_back(last[d]);
    m->dft_gate.push_back(interval[d]);
  }
  return TLM_OK;
}

int tlm_gpu_set_stream(int64_t h, void *stream) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->graph) {
    cudaGraphExecDestroy(m->graph);
    m->graph = nullptr;
  }
  if (m->own_stream && m->stream) cudaStreamDestroy(m->stream);
  m->own_stream = false;
  m->stream = (cudaStream_t)stream;
  if (!stream) {
    CK(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
    m->own_stream = true;
  }
  return TLM_OK;
}

int tlm_gpu_set_timing(int64_t h, int32_t enable) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  m->timing = enable != 0;
  return TLM_OK;
}

int tlm_gpu_run(int64_t h, int32_t first_step, int32_t n_steps) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  CK(cudaSetDevice(m->desc.device));
  int rc = finalize(m);
  if (rc) return rc;
  if (first_step != m->next_step) return fail(TLM_E_STATE, "expected first_step %d, got %d", m->next_step, first_step);
  if (n_steps < 0 || first_step + n_steps - 1 > m->desc.n_timesteps)
    return fail(TLM_E_BADARG, "steps %d..%d beyond n_timesteps %d", first_step, first_step + n_steps - 1, m->desc.n_timesteps);
  if (n_steps == 0) return TLM_OK;
  rc = run_steps(m, n_steps);
  if (rc) return rc;
  m->next_step += n_steps;
  return TLM_OK;
}

static int check_device_error(Mesh *m) {
  if (!m->d_err.p) return TLM_OK;
  int err = 0;
  CK(cudaMemcpy(&err, m->d_err.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (err == tlm::kErrTimeout) return fail(TLM_E_TIMEOUT, "a bulk-copy wait in the cell kernel timed out");
  if (err) return fail(TLM_E_CUDA, "device error word %d", err);
  return TLM_OK;
}

int tlm_gpu_synchronize(int64_t h) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->stream) CK(cudaStreamSynchronize(m->stream));
  return check_device_error(m);
}

int tlm_gpu_set_variant(int64_t h, int32_t variant) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (variant < 0 || variant >= kNumVariants) return fail(TLM_E_BADARG, "variant %d out of range", variant);
  if (m->graph) {
    cudaGraphExecDestroy(m->graph);
    m->graph = nullptr;
  }
  m->variant = variant;
  return TLM_OK;
}

int tlm_gpu_num_variants(int32_t *n) {
  if (!n) return fail(TLM_E_BADARG, "null argument");
  *n = kNumVariants;
  return TLM_OK;
}

int tlm_gpu_last_run_time(int64_t h, float *ms_total, float *ms_cell) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (!m->finalized) return fail(TLM_E_STATE, "no run yet");
  CK(cudaEventSynchronize(m->ev1));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, m->ev0, m->ev1));
  float cell = 0.f;
  for (int s = 0; s < m->timed_steps; s++) {
    float k = 0.f;
    CK(cudaEventElapsedTime(&k, m->kev[2 * s], m->kev[2 * s + 1]));
    cell += k;
  }
  if (ms_total) *ms_total = ms;
  if (ms_cell) *ms_cell = cell;
  return TLM_OK;
}

int tlm_gpu_last_run_launches(int64_t h, int64_t *launches) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  *launches = m->last_launches;
  return TLM_OK;
}

int tlm_gpu_memory_bytes(int64_t h, int64_t *bytes) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  *bytes = (int64_t)m->dev_bytes;
  return TLM_OK;
}

int tlm_gpu_fetch_cell_output(int64_t h, int32_t first, int32_t n, double *out) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->batch_stream) CK(cudaStreamSynchronize(m->batch_stream));
  if (!m->finalized) return fail(TLM_E_STATE, "no run yet");
  if (first < 1 || n < 0 || first + n - 1 >= m->next_step) return fail(TLM_E_BADARG, "steps not yet computed");
  if (m->n_hist == 0 || n == 0) return TLM_OK;
  CK(cudaStreamSynchronize(m->stream));
  const size_t row = (size_t)m->n_hist * 6;
  CK(cudaMemcpy(out, (double *)m->cell_out.p + (size_t)(first - 1) * row, (size_t)n * row * sizeof(double),
                cudaMemcpyDeviceToHost));
  return TLM_OK;
}

int tlm_gpu_fetch_face_output(int64_t h, int32_t first, int32_t n, double *out) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->batch_stream) CK(cudaStreamSynchronize(m->batch_stream));
  if (!m->finalized) return fail(TLM_E_STATE, "no run yet");
  if (first < 1 || n < 0 || first + n - 1 >= m->next_step) return fail(TLM_E_BADARG, "steps not yet computed");
  const size_t nq = m->fpr_face.size();
  if (nq == 0 || n == 0) return TLM_OK;
  CK(cudaStreamSynchronize(m->stream));
  CK(cudaMemcpy(out, (double *)m->fprobe_rec.p + (size_t)(first - 1) * nq, (size_t)n * nq * sizeof(double),
                cudaMemcpyDeviceToHost));
  return TLM_OK;
}

int tlm_gpu_set_far_field(int64_t h, int32_t n, const double *freq, const int32_t *ptr, const int32_t *fout,
                          const int32_t *fcode) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->finalized) return fail(TLM_E_STATE, "tables are fixed after the first run");
  if (n < 0 || (n && (!freq || !ptr || !fout || !fcode))) return fail(TLM_E_BADARG, "bad far-field arguments");
  m->ff_freq.assign(freq, freq + n);
  m->ff_ptr.assign(ptr, ptr + (n ? n + 1 : 0));
  const int ne = n ? ptr[n] : 0;
  for (int d = 0; d < n; d++)
    if (ptr[d] < 0 || ptr[d + 1] < ptr[d]) return fail(TLM_E_BADARG, "far-field face pointers must be non-decreasing");
  m->ff_fout.assign(fout, fout + ne);
  m->ff_fcode.assign(fcode, fcode + ne);
  return TLM_OK;
}

int tlm_gpu_fetch_far_field(int64_t h, double *out) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->batch_stream) CK(cudaStreamSynchronize(m->batch_stream));
  if (!m->finalized) return fail(TLM_E_STATE, "no run yet");
  if (!m->ff_entries) return TLM_OK;
  CK(cudaStreamSynchronize(m->stream));
  CK(cudaMemcpy(out, m->ff_acc.p, (size_t)m->ff_entries * 12 * sizeof(double), cudaMemcpyDeviceToHost));
  return TLM_OK;
}

int tlm_gpu_fetch_dft(int64_t h, double *out) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->batch_stream) CK(cudaStreamSynchronize(m->batch_stream));
  if (!m->finalized) return fail(TLM_E_STATE, "no run yet");
  if (!m->dft_entries) return TLM_OK;
  CK(cudaStreamSynchronize(m->stream));
  CK(cudaMemcpy(out, m->dft_acc.p, (size_t)m->dft_entries * 2 * sizeof(double), cudaMemcpyDeviceToHost));
  return TLM_OK;
}

int tlm_gpu_fetch_links(int64_t h, double *out) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (m->batch_stream) CK(cudaStreamSynchronize(m->batch_stream));
  CK(cudaSetDevice(m->desc.device));
  int rc = finalize(m);
  if (rc) return rc;
  const long long n = (long long)m->desc.nx * m->desc.ny * m->desc.nz;
  DevBuf tmp;
  if ((rc = dalloc(m, tmp, (size_t)n * 12 * sizeof(double)))) return rc;
  const int t_done = m->next_step - 1;
  const int threads = 256;
  const unsigned blocks = (unsigned)((n + threads - 1) / threads);
  if (m->fp64)
    tlm::tlm_gather_links<double><<<blocks, threads, 0, m->stream>>>(mesh_dev<double>(m), t_done, (double *)tmp.p);
  else
    tlm::tlm_gather_links<float><<<blocks, threads, 0, m->stream>>>(mesh_dev<float>(m), t_done, (double *)tmp.p);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(m->stream));
  CK(cudaMemcpy(out, tmp.p, (size_t)n * 12 * sizeof(double), cudaMemcpyDeviceToHost));
  m->dev_bytes -= tmp.bytes;
  return TLM_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free link read-back.
//
// The gather of tlm_gpu_fetch_links needs a device buffer of nx*ny*nz*12
// doubles and gets it with cudaMalloc.  tlm_gpu_fetch_links_noalloc does the
// same gather into a fixed scratch array that lives in the library image
// (file-scope __device__ storage, kNoAllocScratchDoubles doubles = 8 MiB on
// every device that loads the library, held until the process exits), so it
// makes no cudaMalloc/cudaFree call.  In host code the array's name is only a
// host-side stand-in; the device address is looked up once per device with
// cudaGetSymbolAddress, by the first call made on that device.
// ---------------------------------------------------------------------------
namespace {
constexpr size_t kNoAllocScratchDoubles = (size_t)1 << 20;  // 8 MiB
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];
std::mutex g_noalloc_mu;
double *g_noalloc_ptr[64] = {nullptr};
}  // namespace

int tlm_gpu_fetch_links_noalloc(int64_t h, double *out) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (!out) return fail(TLM_E_BADARG, "null output");
  if (!m->finalized)
    return fail(TLM_E_STATE,
                "the mesh has no device state yet: call tlm_gpu_prepare, tlm_gpu_run or tlm_gpu_batch_create first");
  // a mesh inside a batch is advanced on the batch's stream: wait for it, as
  // every other read-back does, so the gather sees the finished steps
  if (m->batch_stream) CK(cudaStreamSynchronize(m->batch_stream));
  const long long n = (long long)m->desc.nx * m->desc.ny * m->desc.nz;
  if ((size_t)n * 12 > kNoAllocScratchDoubles)
    return fail(TLM_E_BADARG, "mesh of %lld cells exceeds the allocation-free read-back limit of %zu cells", n,
                kNoAllocScratchDoubles / 12);
  const int dev = m->desc.device;
  if (dev < 0 || dev >= 64) return fail(TLM_E_BADARG, "device %d out of range", dev);
  CK(cudaSetDevice(dev));
  double *scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
      void *p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p)
        return fail(TLM_E_CUDA, "cudaGetSymbolAddress(scratch) failed on device %d: %s", dev, cudaGetErrorString(e));
      g_noalloc_ptr[dev] = (double *)p;
    }
    scratch = g_noalloc_ptr[dev];
  }
  const int t_done = m->next_step - 1;
  const int threads = 256;
  const unsigned blocks = (unsigned)((n + threads - 1) / threads);
  // every scratch element the caller receives is written by this gather, so
  // nothing has to be cleared first
  if (m->fp64)
    tlm::tlm_gather_links<double><<<blocks, threads, 0, m->stream>>>(mesh_dev<double>(m), t_done, scratch);
  else
    tlm::tlm_gather_links<float><<<blocks, threads, 0, m->stream>>>(mesh_dev<float>(m), t_done, scratch);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, scratch, (size_t)n * 12 * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
  CK(cudaStreamSynchronize(m->stream));
  return TLM_OK;
}

namespace {
// One side of the z-slab halo: the two ports and the storage plane (0 =
// ghost below, 1 = first cell plane, nz = last, nz + 1 = ghost above) of
// the pulses that the last completed step reflected.
int halo_span(Mesh *m, int side, bool put, char **p0, char **p1, size_t *bytes) {
  const size_t esz = m->fp64 ? 8 : 4;
  const int nz = m->desc.nz;
  int z, a, b;
  if (!put) {
    z = side ? nz : 1;
    a = side ? tlm::Vx_zmax : tlm::Vx_zmin;
    b = side ? tlm::Vy_zmax : tlm::Vy_zmin;
  } else {
    z = side ? nz + 1 : 0;
    a = side ? tlm::Vx_zmin : tlm::Vx_zmax;
    b = side ? tlm::Vy_zmin : tlm::Vy_zmax;
  }
  const long long pxpy = (long long)m->Px * m->Py;
  const int t_done = m->next_step - 1;
  char *buf = (char *)m->links.p + ((t_done & 1) ? (size_t)12 * m->plane * esz : 0);
  *p0 = buf + ((size_t)a * m->plane + (size_t)z * pxpy) * esz;
  *p1 = buf + ((size_t)b * m->plane + (size_t)z * pxpy) * esz;
  *bytes = (size_t)pxpy * esz;
  return TLM_OK;
}

int halo_copy(int64_t h, int32_t side, void *dev, bool put) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (!dev) return fail(TLM_E_BADARG, "null halo buffer");
  if (side != 0 && side != 1) return fail(TLM_E_BADARG, "halo side must be 0 (below) or 1 (above)");
  if (m->batch_stream) CK(cudaStreamSynchronize(m->batch_stream));
  CK(cudaSetDevice(m->desc.device));
  int rc = finalize(m);
  if (rc) return rc;
  char *p0, *p1;
  size_t bytes;
  halo_span(m, side, put, &p0, &p1, &bytes);
  char *d = (char *)dev;
  if (put) {
    CK(cudaMemcpyAsync(p0, d, bytes, cudaMemcpyDefault, m->stream));
    CK(cudaMemcpyAsync(p1, d + bytes, bytes, cudaMemcpyDefault, m->stream));
  } else {
    CK(cudaMemcpyAsync(d, p0, bytes, cudaMemcpyDefault, m->stream));
    CK(cudaMemcpyAsync(d + bytes, p1, bytes, cudaMemcpyDefault, m->stream));
  }
  CK(cudaStreamSynchronize(m->stream));
  return TLM_OK;
}
}  // namespace

int tlm_gpu_set_test_wait_pad(int64_t h, int32_t bytes) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (bytes < 0 || bytes > 4096 || bytes % 16)
    return fail(TLM_E_BADARG, "wait pad must be a multiple of 16 bytes in [0, 4096]");
  if (m->graph) {  // the captured launches hold the old value
    cudaGraphExecDestroy(m->graph);
    m->graph = nullptr;
  }
  m->tx_pad = (uint32_t)bytes;
  return TLM_OK;
}

int tlm_gpu_halo_bytes(int64_t h, int64_t *bytes) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  if (!bytes) return fail(TLM_E_BADARG, "null output");
  const size_t esz = m->fp64 ? 8 : 4;
  int rc = finalize(m);  // the padded plane (Px x Py elements) is laid out there
  if (rc) return rc;
  *bytes = (int64_t)(2 * (size_t)m->Px * m->Py * esz);
  return TLM_OK;
}

int tlm_gpu_halo_get(int64_t h, int32_t side, void *dev) { return halo_copy(h, side, dev, false); }

int tlm_gpu_halo_put(int64_t h, int32_t side, const void *dev) { return halo_copy(h, side, (void *)dev, true); }

int tlm_gpu_destroy(int64_t h) {
  std::unique_ptr<Mesh> m;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_meshes.find(h);
    if (it == g_meshes.end()) return fail(TLM_E_BADARG, "bad handle");
    m = std::move(it->second);
    g_meshes.erase(it);
  }
  if (m->stream) cudaStreamSynchronize(m->stream);
  if (m->batch_stream) cudaStreamSynchronize(m->batch_stream);
  return TLM_OK;
}

int tlm_gpu_prepare(int64_t h) {
  Mesh *m = get(h);
  if (!m) return fail(TLM_E_BADARG, "bad handle");
  return finalize(m);
}

int tlm_gpu_pool_release(void) {
  pool::release_all();
  return TLM_OK;
}

int tlm_gpu_pool_cached_bytes(int64_t *bytes) {
  if (!bytes) return fail(TLM_E_BADARG, "null output");
  *bytes = (int64_t)pool::cached_bytes();
  return TLM_OK;
}

int tlm_gpu_last_error(char *buf, int32_t len) {
  if (!buf || len <= 0) return TLM_E_BADARG;
  std::snprintf(buf, (size_t)len, "%s", g_last_error.c_str());
  return TLM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batches: many meshes advanced together by one launch per kernel type.
// ---------------------------------------------------------------------------
namespace {

struct Batch {
  std::vector<int64_t> handles;
  bool fp64 = false;
  int device = 0;
  int variant = 1;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  SideStream side;  // PML / PML-material / special kernels beside the bulk kernel
  bool side_on = false;
  cudaGraphExec_t graph = nullptr;
  std::vector<int> active;  // indices into handles of the current segment
  DevBuf meshes_d, pml_d, faces_d, dfts_d, nsp_d, tiles_d, pmlb_d, spb_d, faceb_d, dftb_d, dbases_d, err_d;
  int n_tiles = 0, n_pmlb = 0, n_spb = 0, n_faceb = 0, n_dftb = 0;
  long long last_cell_updates = 0;
  long long last_launches = 0;
  long long graph_launches = 0;
  size_t dev_bytes = 0;
  ~Batch() {
    if (graph) cudaGraphExecDestroy(graph);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (stream) cudaStreamDestroy(stream);
  }
};

std::map<int64_t, std::unique_ptr<Batch>> g_batches;
int64_t g_next_batch = 1;

Batch *get_batch(int64_t h) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_batches.find(h);
  return it == g_batches.end() ? nullptr : it->second.get();
}

// Upload v into buf on the batch's stream.  A buffer that is large enough
// is overwritten in place: the copy is ordered after the steps already
// queued on that stream, which read the old lists, so a membership change
// between segments needs no device-wide synchronisation (a fresh block
// from the device cache may need one).  A buffer that is too small grows to
// one and a half times what is needed.
template <typename V>
int bupload(Batch *b, DevBuf &buf, const std::vector<V> &v) {
  const size_t need = std::max<size_t>(v.size() * sizeof(V), 16);
  if (!buf.p || buf.cap < need) {
    if (buf.p) b->dev_bytes -= buf.cap;
    cudaError_t e = buf_alloc(buf, need + need / 2);
    if (e != cudaSuccess) return fail(TLM_E_OOM, "device allocation of %zu bytes failed: %s", buf.bytes, cudaGetErrorString(e));
    b->dev_bytes += buf.cap;
  }
  buf.bytes = need;
  if (!v.empty()) CK(cudaMemcpyAsync(buf.p, v.data(), v.size() * sizeof(V), cudaMemcpyHostToDevice, b->stream));
  return TLM_OK;
}

// Build the device work lists of the active meshes.
template <typename T>
int build_batch_lists(Batch *b) {
  const Variant &cf = kVariants[b->variant];
  const int TILE = sizeof(T) == 4 ? cf.tile32 : cf.tile64;
  std::vector<tlm::MeshDev<T>> md;
  std::vector<tlm::PmlList> pl;
  std::vector<tlm::FaceDev> fd;
  std::vector<tlm::DftDev> dd;
  std::vector<int> nsp;
  std::vector<int4> tiles;
  std::vector<int2> pmlb, spb, faceb, dftb;
  std::vector<int *> bases;
  for (size_t a = 0; a < b->active.size(); a++) {
    Mesh *m = get(b->handles[b->active[a]]);
    int rc = build_tiles(m, TILE);
    if (rc) return rc;
    md.push_back(mesh_dev<T>(m));
    pl.push_back(tlm::PmlList{(const unsigned long long *)m->pml_pos.p, (const uint16_t *)m->pml_par16.p,
                              (const int2 *)m->pml_outmap.p, m->n_pml_list, m->n_pml_out, m->pml_shell,
                              m->pml_by_class ? (const double *)m->pml_cls_par.p : nullptr});
    fd.push_back(face_dev(m));
    dd.push_back(dft_dev(m));
    nsp.push_back(m->n_sp_dev);
    for (const int4 &tl : m->host_tiles) tiles.push_back(int4{tl.x, tl.y, tl.z, (int)a});
    for (int s0 = 0; s0 < m->n_pml_list; s0 += 128) pmlb.push_back(int2{(int)a, s0});
    for (int s0 = 0; s0 < m->n_sp_dev; s0 += 128) spb.push_back(int2{(int)a, s0});
    for (int s0 = 0; s0 < (int)m->f_cx.size(); s0 += 128) faceb.push_back(int2{(int)a, s0});
    for (int s0 = 0; s0 < m->dft_entries; s0 += 256) dftb.push_back(int2{(int)a, s0});
    bases.push_back((int *)m->d_base.p);
  }
  b->n_tiles = (int)tiles.size();
  b->n_pmlb = (int)pmlb.size();
  b->n_spb = (int)spb.size();
  b->n_faceb = (int)faceb.size();
  b->n_dftb = (int)dftb.size();
  int rc;
  if ((rc = bupload(b, b->meshes_d, md)) || (rc = bupload(b, b->pml_d, pl)) || (rc = bupload(b, b->faces_d, fd)) ||
      (rc = bupload(b, b->dfts_d, dd)) || (rc = bupload(b, b->nsp_d, nsp)) || (rc = bupload(b, b->tiles_d, tiles)) ||
      (rc = bupload(b, b->pmlb_d, pmlb)) || (rc = bupload(b, b->spb_d, spb)) || (rc = bupload(b, b->faceb_d, faceb)) ||
      (rc = bupload(b, b->dftb_d, dftb)) || (rc = bupload(b, b->dbases_d, bases)))
    return rc;
  return TLM_OK;
}

template <typename T, int VEC, int TILE, int NSTAGE>
int launch_batch_tma(Batch *b, bool dry) {
  using Cfg = tlm::TmaCfg<T, VEC, TILE, NSTAGE>;
  auto kern = tlm::tlm_bulk_tma_kernel<T, VEC, TILE, NSTAGE>;
  CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::SMEM));
  int per_sm = 0, n_sms = 148;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, Cfg::THREADS, Cfg::SMEM));
  CK(cudaDeviceGetAttribute(&n_sms, cudaDevAttrMultiProcessorCount, b->device));
  if (per_sm < 1) per_sm = 1;
  if (dry || !b->n_tiles) return TLM_OK;
  const int grid = std::max(1, std::min(b->n_tiles, per_sm * n_sms));
  tlm::TileList tl{(const int4 *)b->tiles_d.p, b->n_tiles, (int *)b->err_d.p};
  tlm::MeshDev<T> none{};
  kern<<<grid, Cfg::THREADS, Cfg::SMEM, b->stream>>>(none, (const tlm::MeshDev<T> *)b->meshes_d.p, tl, 0);
  b->last_launches++;
  return TLM_OK;
}

template <typename T, int VEC>
int batch_step(Batch *b, bool dry) {
  int rc = TLM_OK;
  if (!dry) {
    for (int i : b->active) {  // set_small_to_zero of the members that ask for it
      Mesh *m = get(b->handles[i]);
      if (m && m->small_every > 0) {
        tlm::tlm_flush_small_kernel<T><<<4 * m->n_sms, 256, 0, b->stream>>>(mesh_dev<T>(m), 0, m->small_every,
                                                                           m->small_value);
        b->last_launches++;
      }
    }
  }
  bool pmm_any = false;
  for (int i : b->active) {
    Mesh *m = get(b->handles[i]);
    if (m && m->n_pmm) pmm_any = true;
  }
  const bool side = !dry && b->side_on && (b->n_pmlb || b->n_spb || pmm_any);
  if (side && (rc = b->side.begin(b->stream))) return rc;
  if constexpr (sizeof(T) == 4) {
    switch (b->variant) {
      case 1: rc = launch_batch_tma<T, VEC, 1024, 2>(b, dry); break;
      case 2: rc = launch_batch_tma<T, VEC, 512, 3>(b, dry); break;
      case 3: rc = launch_batch_tma<T, VEC, 512, 4>(b, dry); break;
      case 4: rc = launch_batch_tma<T, VEC, 1024, 3>(b, dry); break;
      default: rc = launch_batch_tma<T, VEC, 256, 6>(b, dry); break;
    }
  } else {
    switch (b->variant) {
      case 1: rc = launch_batch_tma<T, VEC, 512, 2>(b, dry); break;
      case 2: rc = launch_batch_tma<T, VEC, 256, 3>(b, dry); break;
      case 3: rc = launch_batch_tma<T, VEC, 256, 4>(b, dry); break;
      case 4: rc = launch_batch_tma<T, VEC, 512, 3>(b, dry); break;
      default: rc = launch_batch_tma<T, VEC, 128, 6>(b, dry); break;
    }
  }
  if (rc || dry) return rc;
  tlm::BatchDev<T> bd{};
  bd.meshes = (const tlm::MeshDev<T> *)b->meshes_d.p;
  bd.pml = (const tlm::PmlList *)b->pml_d.p;
  bd.faces = (const tlm::FaceDev *)b->faces_d.p;
  bd.dfts = (const tlm::DftDev *)b->dfts_d.p;
  bd.n_special = (const int *)b->nsp_d.p;
  bd.pml_blocks = (const int2 *)b->pmlb_d.p;
  bd.special_blocks = (const int2 *)b->spb_d.p;
  bd.face_blocks = (const int2 *)b->faceb_d.p;
  bd.dft_blocks = (const int2 *)b->dftb_d.p;
  bd.n_pml_blocks = b->n_pmlb;
  bd.n_special_blocks = b->n_spb;
  bd.n_face_blocks = b->n_faceb;
  bd.n_dft_blocks = b->n_dftb;
  bd.d_bases = (int *const *)b->dbases_d.p;
  bd.n_active = (int)b->active.size();
  const cudaStream_t ss = side ? b->side.s : b->stream;
  if (b->n_pmlb) { tlm::tlm_pml_batch_kernel<T><<<b->n_pmlb, 128, 0, ss>>>(bd, 0); b->last_launches++; }
  for (int i : b->active) {  // PML cells inside materials of the members that have them
    Mesh *m = get(b->handles[i]);
    if (m && m->n_pmm) {
      tlm::tlm_pml_material_kernel<T><<<(m->n_pmm + 127) / 128, 128, 0, ss>>>(mesh_dev<T>(m), pmm_list(m), 0);
      b->last_launches++;
    }
  }
  if (b->n_spb) {
    int maxo = 0;
    for (int i : b->active) {
      Mesh *m = get(b->handles[i]);
      if (m) maxo = std::max(maxo, std::max(m->filt_eo, m->filt_mo));
    }
    switch (special_order_bound(maxo)) {
      case 1: tlm::tlm_special_batch_kernel<T, 1><<<b->n_spb, 128, 0, ss>>>(bd, 0); break;
      case 2: tlm::tlm_special_batch_kernel<T, 2><<<b->n_spb, 128, 0, ss>>>(bd, 0); break;
      case 3: tlm::tlm_special_batch_kernel<T, 3><<<b->n_spb, 128, 0, ss>>>(bd, 0); break;
      case 4: tlm::tlm_special_batch_kernel<T, 4><<<b->n_spb, 128, 0, ss>>>(bd, 0); break;
      default: tlm::tlm_special_batch_kernel<T, tlm::kMaxOrder><<<b->n_spb, 128, 0, ss>>>(bd, 0); break;
    }
    b->last_launches++;
  }
  if (side && (rc = b->side.end(b->stream))) return rc;
  for (int i : b->active) {  // SAR volumes of the members that have them
    Mesh *m = get(b->handles[i]);
    if (m && m->sar_entries) {
      const tlm::SarDev sd = sar_dev(m);
      tlm::tlm_sar_kernel<<<(sd.n_entries + 255) / 256, 256, 0, b->stream>>>(sd, (const int *)m->d_base.p, 0);
      b->last_launches++;
    }
  }
  for (int i : b->active) {  // time-domain output volumes of the members that have them
    Mesh *m = get(b->handles[i]);
    if (m && !m->ovol_gate.empty()) {
      const tlm::OutVolDev ov = out_vol_dev(m);
      tlm::tlm_output_volume_kernel<<<ov.n_vol, tlm::kOutVolThreads, 0, b->stream>>>(ov, (const int *)m->d_base.p, 0);
      b->last_launches++;
    }
  }
  for (int i : b->active) {  // frequency output volumes of the members that have them
    Mesh *m = get(b->handles[i]);
    if (m && m->vdft_entries) {
      const tlm::VolDftDev vd = vol_dft_dev(m);
      tlm::tlm_volume_dft_kernel<<<(vd.n_entries + 255) / 256, 256, 0, b->stream>>>(vd, (const int *)m->d_base.p, 0);
      b->last_launches++;
    }
  }
  if (b->n_faceb) { tlm::tlm_face_batch_kernel<T><<<b->n_faceb, 128, 0, b->stream>>>(bd, 0); b->last_launches++; }
  for (int i : b->active) {  // outer-boundary Huygens surfaces of the members that have them
    Mesh *m = get(b->handles[i]);
    if (m && m->hs_outer && m->hs_n) {
      tlm::tlm_outer_huygens_kernel<T><<<(m->hs_n + 127) / 128, 128, 0, b->stream>>>(mesh_dev<T>(m), outer_hs_dev(m), 0);
      b->last_launches++;
    }
  }
  for (int i : b->active) {  // far-field surfaces of the members that have them
    Mesh *m = get(b->handles[i]);
    if (m && m->ff_entries) {
      const tlm::FarFieldDev fdv = far_field_dev(m);
      tlm::tlm_far_field_kernel<<<(fdv.n_entries + 255) / 256, 256, 0, b->stream>>>(fdv, (const int *)m->d_base.p, 0);
      b->last_launches++;
    }
  }
  for (int i : b->active) {  // face output points of the members that have them
    Mesh *m = get(b->handles[i]);
    if (m && !m->fpr_face.empty()) {
      const tlm::FaceProbeDev pd = face_probe_dev(m);
      tlm::tlm_face_probe_kernel<<<(pd.n + 127) / 128, 128, 0, b->stream>>>(pd, (const double *)m->face_field.p,
                                                                             (const int *)m->d_base.p, 0);
      b->last_launches++;
    }
  }
  for (int i : b->active) {  // power surfaces and mode outputs of the members that have them
    Mesh *m = get(b->handles[i]);
    if (m && m->ps_entries) {
      const tlm::PowerSurfDev pd2 = power_surf_dev(m);
      tlm::tlm_power_surface_kernel<<<(pd2.n_entries + 255) / 256, 256, 0, b->stream>>>(pd2, (const int *)m->d_base.p,
                                                                                       0);
      b->last_launches++;
    }
    if (m && !m->mode_comp.empty()) {
      const tlm::ModeDev mdv = mode_dev(m);
      tlm::tlm_mode_kernel<<<mdv.n_modes, tlm::kOutVolThreads, 0, b->stream>>>(mdv, (const int *)m->d_base.p, 0);
      b->last_launches++;
    }
  }
  for (int i : b->active) {  // RCS surfaces of the members that have them
    Mesh *m = get(b->handles[i]);
    if (m && m->rcs_on && !m->rcs_fout.empty()) {
      const tlm::RcsDev rd = rcs_dev(m);
      tlm::tlm_rcs_kernel<<<(rd.n_faces + 255) / 256, 256, 0, b->stream>>>(rd, (const int *)m->d_base.p, 0);
      b->last_launches++;
    }
  }
  for (int i : b->active) {  // time-domain output surfaces of the members that have them
    Mesh *m = get(b->handles[i]);
    if (m && m->osurf_entries) {
      const tlm::OutSurfDev od = out_surf_dev(m);
      tlm::tlm_output_surface_kernel<<<(od.n_entries + 255) / 256, 256, 0, b->stream>>>(od, (const int *)m->d_base.p,
                                                                                        0);
      b->last_launches++;
    }
  }
  if (b->n_dftb) { tlm::tlm_dft_batch_kernel<T><<<b->n_dftb, 256, 0, b->stream>>>(bd, 0); b->last_launches++; }
  tlm::tlm_advance_batch<<<(bd.n_active + 127) / 128, 128, 0, b->stream>>>(bd.d_bases, bd.n_active, 1);
  b->last_launches++;
  CK(cudaGetLastError());
  return TLM_OK;
}

int batch_step_any(Batch *b, bool dry) { return b->fp64 ? batch_step<double, 2>(b, dry) : batch_step<float, 4>(b, dry); }

}  // namespace

extern "C" {

int tlm_gpu_batch_create(const int64_t *handles, int32_t n, int64_t *batch) {
  if (!handles || n < 1 || !batch) return fail(TLM_E_BADARG, "bad batch arguments");
  auto b = std::make_unique<Batch>();
  for (int i = 0; i < n; i++) {
    Mesh *m = get(handles[i]);
    if (!m) return fail(TLM_E_BADARG, "bad handle at position %d", i);
    if (m->batch_stream) return fail(TLM_E_STATE, "mesh %d already belongs to a batch", i);
    if (i == 0) {
      b->fp64 = m->fp64;
      b->device = m->desc.device;
    } else if (m->fp64 != b->fp64 || m->desc.device != b->device) {
      return fail(TLM_E_BADARG, "all meshes of a batch need the same precision and device");
    }
    for (int j = 0; j < i; j++)
      if (handles[j] == handles[i]) return fail(TLM_E_BADARG, "mesh listed twice");
  }
  CK(cudaSetDevice(b->device));
  for (int i = 0; i < n; i++) {
    Mesh *m = get(handles[i]);
    int rc = finalize(m);
    if (rc) return rc;
    if (m->stream) CK(cudaStreamSynchronize(m->stream));
  }
  b->handles.assign(handles, handles + n);
  CK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  CK(cudaEventCreate(&b->ev0));
  CK(cudaEventCreate(&b->ev1));
  b->side_on = side_stream_enabled(0, true);
  if (b->side_on) {
    int rc = b->side.init();
    if (rc) return rc;
  }
  {
    std::vector<int> zero(1, 0);
    int rc = bupload(b.get(), b->err_d, zero);
    if (rc) return rc;
  }
  for (int i = 0; i < n; i++) get(handles[i])->batch_stream = b->stream;
  std::lock_guard<std::mutex> lk(g_mu);
  const int64_t h = g_next_batch++;
  g_batches[h] = std::move(b);
  *batch = h;
  return TLM_OK;
}

int tlm_gpu_batch_set_variant(int64_t bh, int32_t variant) {
  Batch *b = get_batch(bh);
  if (!b) return fail(TLM_E_BADARG, "bad batch handle");
  if (variant < 1 || variant >= kNumVariants) return fail(TLM_E_BADARG, "batch variant must be a TMA variant (1..%d)", kNumVariants - 1);
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  b->variant = variant;
  b->active.clear();  // forces a rebuild of the work lists
  return TLM_OK;
}

int tlm_gpu_batch_run(int64_t bh, int32_t n_steps) {
  Batch *b = get_batch(bh);
  if (!b) return fail(TLM_E_BADARG, "bad batch handle");
  if (n_steps < 0) return fail(TLM_E_BADARG, "negative step count");
  CK(cudaSetDevice(b->device));
  b->last_launches = 0;
  b->last_cell_updates = 0;
  CK(cudaEventRecord(b->ev0, b->stream));
  int left = n_steps;
  while (left > 0) {
    std::vector<int> act;
    int seg = left;
    for (size_t i = 0; i < b->handles.size(); i++) {
      Mesh *m = get(b->handles[i]);
      const int rem = m->desc.n_timesteps - m->next_step + 1;
      if (rem > 0) {
        act.push_back((int)i);
        seg = std::min(seg, rem);
      }
    }
    if (act.empty()) break;
    if (act != b->active) {
      b->active = act;
      int rc = b->fp64 ? build_batch_lists<double>(b) : build_batch_lists<float>(b);
      if (rc) return rc;
      if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
      }
    }
    if (!b->graph) {
      int rc = batch_step_any(b, true);  // kernel attributes outside capture
      if (rc) return rc;
      cudaGraph_t g;
      CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      const long long saved = b->last_launches;
      rc = batch_step_any(b, false);
      cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
      if (rc) return rc;
      if (ce != cudaSuccess) return fail(TLM_E_CUDA, "batch graph capture: %s", cudaGetErrorString(ce));
      ce = cudaGraphInstantiate(&b->graph, g, 0);
      cudaGraphDestroy(g);
      if (ce != cudaSuccess) return fail(TLM_E_CUDA, "batch graph instantiate: %s", cudaGetErrorString(ce));
      b->graph_launches = b->last_launches - saved;
      b->last_launches = saved;
    }
    for (int k = 0; k < seg; k++) {
      CK(cudaGraphLaunch(b->graph, b->stream));
      b->last_launches += b->graph_launches;
    }
    for (int i : b->active) {
      Mesh *m = get(b->handles[i]);
      m->next_step += seg;
      b->last_cell_updates += (long long)seg * m->desc.nx * m->desc.ny * m->desc.nz;
    }
    left -= seg;
  }
  CK(cudaEventRecord(b->ev1, b->stream));
  return TLM_OK;
}

int tlm_gpu_batch_set_members(int64_t bh, const int64_t *handles, int32_t n) {
  Batch *b = get_batch(bh);
  if (!b) return fail(TLM_E_BADARG, "bad batch handle");
  if (!handles || n < 1) return fail(TLM_E_BADARG, "bad batch arguments");
  for (int i = 0; i < n; i++) {
    Mesh *m = get(handles[i]);
    if (!m) return fail(TLM_E_BADARG, "bad handle at position %d", i);
    const bool member = std::find(b->handles.begin(), b->handles.end(), handles[i]) != b->handles.end();
    if (m->batch_stream && !member) return fail(TLM_E_STATE, "mesh %d belongs to another batch", i);
    if (m->fp64 != b->fp64 || m->desc.device != b->device)
      return fail(TLM_E_BADARG, "all meshes of a batch need the same precision and device");
    for (int j = 0; j < i; j++)
      if (handles[j] == handles[i]) return fail(TLM_E_BADARG, "mesh listed twice");
  }
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  for (int i = 0; i < n; i++) {
    Mesh *m = get(handles[i]);
    int rc = finalize(m);
    if (rc) return rc;
    if (m->stream) CK(cudaStreamSynchronize(m->stream));
  }
  for (int64_t h : b->handles) {  // leavers run alone again
    Mesh *m = get(h);
    if (m && std::find(handles, handles + n, h) == handles + n) m->batch_stream = nullptr;
  }
  b->handles.assign(handles, handles + n);
  for (int i = 0; i < n; i++) get(handles[i])->batch_stream = b->stream;
  b->active.clear();  // the next run rebuilds the work lists and the graph
  return TLM_OK;
}

int tlm_gpu_batch_synchronize(int64_t bh) {
  Batch *b = get_batch(bh);
  if (!b) return fail(TLM_E_BADARG, "bad batch handle");
  CK(cudaStreamSynchronize(b->stream));
  int err = 0;
  CK(cudaMemcpy(&err, b->err_d.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (err == tlm::kErrTimeout) return fail(TLM_E_TIMEOUT, "a bulk-copy wait in the batched cell kernel timed out");
  return TLM_OK;
}

int tlm_gpu_batch_last_run(int64_t bh, float *ms, int64_t *cell_updates, int64_t *launches) {
  Batch *b = get_batch(bh);
  if (!b) return fail(TLM_E_BADARG, "bad batch handle");
  CK(cudaEventSynchronize(b->ev1));
  float t = 0.f;
  CK(cudaEventElapsedTime(&t, b->ev0, b->ev1));
  if (ms) *ms = t;
  if (cell_updates) *cell_updates = b->last_cell_updates;
  if (launches) *launches = b->last_launches;
  return TLM_OK;
}

int tlm_gpu_batch_destroy(int64_t bh) {
  std::unique_ptr<Batch> b;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_batches.find(bh);
    if (it == g_batches.end()) return fail(TLM_E_BADARG, "bad batch handle");
    b = std::move(it->second);
    g_batches.erase(it);
  }
  cudaStreamSynchronize(b->stream);
  for (int64_t h : b->handles) {
    Mesh *m = get(h);
    if (m) m->batch_stream = nullptr;
  }
  return TLM_OK;
}

}  // extern "C"
