// A stand-alone C++ caller of the library's C ABI (include/tlm_gpu.h), used
// by tests/test_capi_driver.py.  It makes the calls a Fortran driver makes
// in place of run_TLM (SRC/GGI_TLM.F90:157), in the same order, from plain
// arrays, with no Python or torch in the process:
//   create -> set_cells -> set_materials -> set_pml -> set_excitation ->
//   set_faces -> set_huygens -> set_outputs -> set_face_excitation ->
//   set_face_outputs -> set_dft -> (run 100 steps, fetch the output points)
//   ... -> fetch_dft -> destroy,
// and stops with the library's message and exit code 1 on the first error,
// as the Fortran shim does (write(*,*) msg; STOP 1).
//
//   capi_driver <table dir> <out dir> <precision 32|64>
//
// The table directory holds manifest.txt with one line per entry,
// "<name> i <count>" (int32 file <name>.bin), "<name> d <count>" (float64
// file <name>.bin) or "<name> s <value>" (a scalar), written from the
// problem tables by the test.  The output directory receives cell_out.bin
// ([steps][n_kept][6]), face_out.bin ([steps][n_face_points]) and dft.bin.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../include/tlm_gpu.h"

namespace {

struct Tables {
  std::map<std::string, std::vector<int32_t>> i;
  std::map<std::string, std::vector<double>> d;
  std::map<std::string, double> s;

  template <typename V>
  static bool read_bin(const std::string &path, std::vector<V> &v, size_t n) {
    v.assign(n ? n : 1, V(0));
    if (!n) return true;
    std::ifstream f(path, std::ios::binary);
    return f && f.read(reinterpret_cast<char *>(v.data()), (std::streamsize)(n * sizeof(V)));
  }

  bool load(const std::string &dir) {
    std::ifstream m(dir + "/manifest.txt");
    if (!m) return false;
    std::string line;
    while (std::getline(m, line)) {
      std::istringstream ls(line);
      std::string name, kind;
      if (!(ls >> name >> kind)) continue;
      if (kind == "s") {
        double v;
        ls >> v;
        s[name] = v;
      } else {
        size_t n = 0;
        ls >> n;
        const std::string p = dir + "/" + name + ".bin";
        if (kind == "i" ? !read_bin(p, i[name], n) : !read_bin(p, d[name], n)) {
          std::fprintf(stderr, "cannot read %s\n", p.c_str());
          return false;
        }
      }
    }
    return true;
  }
  const int32_t *ip(const std::string &k) { return i.at(k).data(); }
  const double *dp(const std::string &k) { return d.at(k).data(); }
  int32_t n(const std::string &k) { return (int32_t)s.at(k); }
  bool has(const std::string &k) { return s.count(k) && s.at(k) != 0.0; }
};

bool write_bin(const std::string &path, const std::vector<double> &v) {
  std::ofstream f(path, std::ios::binary);
  return f && f.write(reinterpret_cast<const char *>(v.data()), (std::streamsize)(v.size() * sizeof(double)));
}

}  // namespace

// The shim's error handling: print the library's message and stop.
#define CALL(expr)                                                        \
  do {                                                                    \
    const int rc_ = (expr);                                               \
    if (rc_ != 0) {                                                       \
      char msg_[512];                                                     \
      tlm_gpu_last_error(msg_, (int32_t)sizeof(msg_));                    \
      std::fprintf(stderr, "ERROR in run_TLM_gpu: %s (%d)\n", msg_, rc_); \
      return 1;                                                           \
    }                                                                     \
  } while (0)

int main(int argc, char **argv) {
  if (argc != 4) {
    std::fprintf(stderr, "usage: capi_driver <table dir> <out dir> <precision 32|64>\n");
    return 2;
  }
  Tables t;
  if (!t.load(argv[1])) {
    std::fprintf(stderr, "cannot load the tables in %s\n", argv[1]);
    return 2;
  }
  const std::string out = argv[2];
  tlm_gpu_mesh_desc desc{};
  desc.nx = t.n("nx");
  desc.ny = t.n("ny");
  desc.nz = t.n("nz");
  desc.n_timesteps = t.n("n_timesteps");
  desc.dl = t.s.at("dl");
  desc.dt = t.s.at("dt");
  for (int k = 0; k < 6; k++) desc.R[k] = t.dp("R")[k];
  desc.precision = std::atoi(argv[3]) == 32 ? TLM_PRECISION_FP32 : TLM_PRECISION_FP64;
  desc.device = 0;
  int64_t h = 0;
  CALL(tlm_gpu_create(&desc, &h));
  CALL(tlm_gpu_set_cells(h, t.ip("cell_code"), t.n("n_special"), t.ip("sp_material"), t.ip("sp_pml"),
                         t.ip("sp_excitation"), t.ip("sp_output")));
  if (t.has("n_materials"))
    CALL(tlm_gpu_set_materials(h, t.n("n_materials"), t.ip("mat_type"), t.ip("mat_eps_exists"), t.ip("mat_mu_exists"),
                               t.ip("mat_eps_order"), t.ip("mat_mu_order"), t.dp("mat_Ys_eps_f"), t.dp("mat_Zs_mu_f"),
                               t.dp("mat_Ge"), t.dp("mat_Rm"), t.dp("mat_eps_a"), t.dp("mat_eps_b"), t.dp("mat_mu_a"),
                               t.dp("mat_mu_b"), t.n("mat_stride")));
  CALL(tlm_gpu_set_pml(h, t.n("n_pml_params"), t.dp("pml_params"), t.n("n_pml_cells"), t.ip("pml_cell_param")));
  CALL(tlm_gpu_set_excitation(h, t.n("n_functions"), t.n("n_timesteps"), t.dp("fn_value"), t.dp("fn_value_face"),
                              t.n("n_exc_points"), t.ip("pt_cell"), t.ip("pt_comp"), t.ip("pt_fn"), t.ip("pt_type"),
                              t.n("n_exc_cells")));
  CALL(tlm_gpu_set_faces(h, t.n("n_faces"), t.ip("face_cx"), t.ip("face_cy"), t.ip("face_cz"), t.ip("face_dir"),
                         t.ip("face_exc"), t.ip("face_out"), t.n("n_exc_faces"), t.n("n_out_faces")));
  if (t.has("hs_n"))
    CALL(tlm_gpu_set_huygens(h, t.n("hs_n"), t.ip("hs_face_exc"), t.ip("hs_norm"), t.dp("hs_offset"), t.dp("hs_Ei"),
                             t.dp("hs_Hi"), t.s.at("hs_offset_min"), t.s.at("hs_c"), t.n("hs_fn")));
  CALL(tlm_gpu_set_outputs(h, t.n("n_out_cells")));
  if (t.has("n_face_points"))
    CALL(tlm_gpu_set_face_excitation(h, t.n("n_face_points"), t.ip("fpt_face"), t.ip("fpt_comp"), t.ip("fpt_fn"),
                                     t.ip("fpt_type")));
  if (t.has("n_face_probes"))
    CALL(tlm_gpu_set_face_outputs(h, t.n("n_face_probes"), t.ip("fprobe_face"), t.ip("fprobe_side"),
                                  t.ip("fprobe_comp")));
  if (t.has("n_dft"))
    CALL(tlm_gpu_set_dft(h, t.n("n_dft"), t.dp("dft_freq"), t.ip("dft_comp"), t.ip("dft_face_ptr"),
                         t.ip("dft_face_out"), t.ip("dft_face_side")));
  if (t.has("n_dft"))  // the surfaces' output steps (every step unless the input gives a timing block)
    CALL(tlm_gpu_set_dft_gate(h, t.n("n_dft"), t.ip("dft_first"), t.ip("dft_last"), t.ip("dft_interval")));
  // the time loop, in chunks: after each chunk the output points are read
  // back (where the Fortran shim writes its .tout lines)
  const int n_steps = desc.n_timesteps, chunk = 100;
  const size_t n_kept = (size_t)t.n("n_kept"), n_fp = (size_t)t.n("n_face_probes");
  std::vector<double> cell_out, face_out;
  for (int first = 1; first <= n_steps; first += chunk) {
    const int n = first + chunk - 1 <= n_steps ? chunk : n_steps - first + 1;
    CALL(tlm_gpu_run(h, first, n));
    std::vector<double> c((size_t)n * n_kept * 6 + 1), f((size_t)n * n_fp + 1);
    CALL(tlm_gpu_fetch_cell_output(h, first, n, c.data()));
    CALL(tlm_gpu_fetch_face_output(h, first, n, f.data()));
    cell_out.insert(cell_out.end(), c.begin(), c.begin() + (ptrdiff_t)((size_t)n * n_kept * 6));
    face_out.insert(face_out.end(), f.begin(), f.begin() + (ptrdiff_t)((size_t)n * n_fp));
  }
  const size_t n_dft_faces = t.has("n_dft") ? (size_t)t.ip("dft_face_ptr")[t.n("n_dft")] : 0;
  std::vector<double> dft(2 * n_dft_faces + 2);
  CALL(tlm_gpu_fetch_dft(h, dft.data()));
  dft.resize(2 * n_dft_faces);
  CALL(tlm_gpu_destroy(h));
  if (!write_bin(out + "/cell_out.bin", cell_out) || !write_bin(out + "/face_out.bin", face_out) ||
      !write_bin(out + "/dft.bin", dft)) {
    std::fprintf(stderr, "cannot write the results to %s\n", out.c_str());
    return 2;
  }
  std::printf("ok %d steps\n", n_steps);
  return 0;
}
