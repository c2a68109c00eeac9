// rbmd_force.cu -- C ABI and host driver of the B200 force path (see include/rbmd_force.h).
//
// The driver reproduces the dispatch of ExecutionNVT::ComputeAllForce
// (rbmd/framework/run/ExecutionNVT.cpp:185-222) and the step order of ExecutionNVT::Solve
// (:133-159) on top of the sm_100a kernels in kernels_*.cuh.  All work of one call is queued on
// the caller's stream (k-space structure factors on a forked side stream that joins before the
// force pass); host synchronisation happens only where a call must return host data or check
// the list capacity.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <random>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <mutex>
#include <set>
#include <sstream>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "../../include/rbmd_force.h"
#include "common.cuh"
#include "eam_funcfl.hpp"
#include "json.hpp"
#include "kernels_cells.cuh"
#include "kernels_force.cuh"
#include "kernels_md.cuh"
#include "kernels_rbl.cuh"
#include "kernels_learned.cuh"
#include "proposal.hpp"

using namespace rbmd;

namespace {

constexpr int kKL = 2;           // k samples per lane in the structure-factor kernel
constexpr int kStageBytes = 48 * 1024;   // shared memory for k staging in the force pass
constexpr int kSamplerD = 640;   // pre-drawn proposals per axis in the sampler kernel (38 KB smem)
constexpr int kMdChunk = 2048;   // atoms per kinetic-energy chunk

}  // namespace

namespace rbmd_internal {
char g_last_error[512] = "";
}
using rbmd_internal::g_last_error;

namespace {

#define CK(x)                                                                            \
  do {                                                                                   \
    cudaError_t e_ = (x);                                                                \
    if (e_ != cudaSuccess) {                                                             \
      std::snprintf(g_last_error, sizeof g_last_error, "%s:%d %s: %s", __FILE__, __LINE__, \
                    #x, cudaGetErrorString(e_));                                         \
      return RBMD_ERR_CUDA;                                                              \
    }                                                                                    \
  } while (0)

template <class T>
cudaError_t dalloc(T** p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  return cudaMalloc((void**)p, count * sizeof(T));
}
template <class T>
void dfree(T*& p) {
  if (p) cudaFree((void*)p);
  p = nullptr;
}

struct Units { double kB, fmt2v, mvv2e, qqr2e; };

// ExecutionMD::InitParameters (rbmd/framework/run/ExecutionMD.cpp:328-353)
Units units_for(const std::string& u) {
  if (u == "REAL") return {1.9872067e-3, 4.186e-4, 1.0 / 4.186e-4, 332.06371};
  if (u == "METAL") return {8.617343e-5, 1.0 / 1.0364269e-4, 1.0364269e-4, 14.399645};
  return {1.0, 1.0, 1.0, 1.0};
}

}  // namespace

struct rbmd_force {
  // ---------------- configuration ----------------
  std::string ff = "LJ/CUT", nbr_type = "VERLETLIST", coul_type = "RBE", unit = "LJ";
  std::string shake = "null", init_way = "read_data", tctrl = "";
  bool far = false, fp64 = false;
  double rc = 2.5, rs = 2.5, skin = 0.0, alpha = 0.1;
  double rbl_sample_num = 100;   // neighbor.neighbor_sample_num (RBL)
  bool rbl_table = false;        // compat.rbl_erf_table: G from the reference's alpha=0.1 table
  bool rbl_shell_coul = true;    // !compat.rbl_drop_shell_coulomb
  bool eam_ref_sign = false;     // compat.eam_verlet_pair_vector: reference's reversed EAM force
  // k-proposal of the RBE sampler: "gauss" (the reference's Metropolis-Hastings chain over the
  // Gaussian), "gauss_iid" (exact independent draws from the same Gaussian) or "learned" (the
  // Gaussian reweighted per |k| bin by the network, importance weights p/q; until trained or
  // given parameters it draws from the Gaussian with unit weights)
  std::string proposal = "gauss";
  bool prop_trained = false;
  PropRep* d_prep = nullptr;
  int prop_stage_bytes = 0;            // shared memory of k_prop_sample (largest replica's CDFs)
  std::vector<PropRep> prep_h;
  double* d_cdf = nullptr;
  double* d_wbin = nullptr;         // [nrep][256] Gaussian mass per bin
  std::vector<double> wbin_h;
  double* d_pw = nullptr;           // [Ptot] importance weights of the drawn samples
  float *d_mlp = nullptr, *d_mlp_t = nullptr, *d_h = nullptr, *d_spec = nullptr;   // d_mlp_t: k_mlp_prep layout
  int* d_spec_init = nullptr;
  int P = 100, kmax = 2;
  unsigned long long seed = 20240101ull;
  Units u{1, 1, 1, 1};
  double dt = 0.005, T0 = 1.0, Tdamp = 1.0;
  int tstat = 0, dof_mode = 0;
  double near_coul_scale = 1.0;
  double shake_tol = 1e-5;
  int energy_every = 0;   // energies inside step(): every outputs.thermo_out.interval steps
  int cap_override = 0;   // neighbor.capacity: initial list capacity (grown on overflow)
  int tpa_list = 0, tpa_near = 128;
  int rbl_list_warp = -1;               // RBL list build: 1 one warp per atom, 0 one thread per atom, -1 by size
  int rbl_lanes = 0;                    // RBL force pass lanes per atom (0: by size)
  int num_sms = 148;                    // SMs of the bound device (cudaDevAttrMultiProcessorCount)
  int near_variant = 1;                 // 1: k_near_lean where it applies (lean_ok), 0: k_near_force
  int near_lanes = 1;                   // near pass lanes per atom: 1, or 4 / 8 / 16 / 32     // list build: 0 = staged kernel, else threads per block of
                                        // k_nlist; threads per block of the force pass
  bool autotune = false;                // "autotune": true tunes them at the first compute
  bool tuned = false;
  bool list_valid = false;   // a list (and x_ref) exists from an earlier build
  int shake_max_iter = 5000;
  std::string potential_file, potential_format;   // format: "", "funcfl" or "setfl"

  // ---------------- replicas ----------------
  int nrep = 1;
  std::vector<rbmd_box> boxes;
  std::vector<RepDev> reps_h;
  int ncell_total = 0, num_cycles = 1;

  // ---------------- per-type LJ ----------------
  int ntypes = 1;          // declared types (atom type ids must lie below)
  int nt_eff = 1;          // 1 when every type pair has the same LJ coefficients
  LJTable ljt_h{};
  bool have_pair_coeffs = false;

  // ---------------- EAM ----------------
  FuncflTables eam_h;
  bool eam_loaded = false;

  // ---------------- water ----------------
  int64_t n_mol = 0;
  std::vector<int32_t> hoh_h;
  double bond_k = 0, bond_r0 = 1, angle_k = 0, angle_t0 = 109.47;

  // ---------------- general CVFF topology (rbmd_force_set_topology) ----------------
  bool topo = false;                 // bonded terms of a topology replace the water extras
  bool special = false;              // hyper_parameters.extend.special_bonds given
  double special_w[3] = {0, 0, 0};
  int64_t topo_n = 0;
  int topo_nb = 0, topo_na = 0, topo_nd = 0;
  std::vector<int32_t> term_atom_h, tmult_h, sc_off_h, sc_id_h, row_off_h, row_idx_h, sp_off_h, sp_id_h,
      comp_h;
  std::vector<double> tk_h, ta_h, sc_fac_h, sp_w_h;

  // ---------------- bound atoms ----------------
  rbmd_atoms_dev at{};
  std::vector<int64_t> rep_off;
  bool bound = false;
  int n = 0, stride = 0, cap = 0;
  double sum_q2 = 0;

  // ---------------- device buffers ----------------
  RepDev* d_reps = nullptr;
  LJTable* d_ljt = nullptr;
  int *d_rep_of = nullptr, *d_cell_of = nullptr, *d_cell_count = nullptr, *d_cell_start = nullptr,
      *d_cursor = nullptr, *d_tmp = nullptr, *d_slot_atom = nullptr, *d_atom_slot = nullptr;
  void* d_pos4 = nullptr;
  void* d_frac = nullptr;
  int2* d_meta = nullptr;
  int *d_nbr = nullptr, *d_count = nullptr, *d_maxcount = nullptr;
  // RBL: rows [0, core_cap) of d_nbr hold the core list (counts in d_count), rows
  // [core_cap, cap) the kept shell pairs (counts in d_count2); rbl_sizes_h = rs_num, rc_num, pice
  // of the reference's sizing formulas for replica 0
  int* d_count2 = nullptr;
  int core_cap = 0, shell_cap = 0;
  int64_t rbl_sizes_h[3] = {0, 0, 0};
  double* d_mean_partial = nullptr;
  float* d_erf_tab = nullptr;   // compat.rbl_erf_table
  int *d_rebuild = nullptr, *d_block_sums = nullptr;   // d_rebuild[nrep + 1]: per replica, then any
  int* d_cell_rep = nullptr;                            // replica of each cell (batches only)
  unsigned long long* d_nbuilds = nullptr;
  ListSeg* d_segs = nullptr;   // staged list build: one block per segment of a cell row
  int nsegs = 0, stage_cap = 0;
  double* d_xref = nullptr;
  uint32_t* d_status = nullptr;
  double* d_eslot = nullptr;   // 2 per slot (lj, coul)
  double* d_esum = nullptr;    // scratch sums
  // RBE
  int Ptot = 0, nitems = 0, rho_threads = 64, ktile = 128, kstage = 0;
  bool minimg = true, want_energy = true;
  bool kspace_priority = true;
  bool orig_pred = false;        // neighbor.type "ORIGINAL": pair predicate d^2 < rc^2   // execution.kspace_priority: side stream at the highest priority
  int* d_krep = nullptr;
  int nq = 0;               // charged atoms (the k-space path runs over these only)
  int* d_qidx = nullptr;
  void* d_krec = nullptr;
  int* d_kvec = nullptr;
  RhoItem* d_items = nullptr;
  RhoRep* d_rhorep = nullptr;
  void* d_partial = nullptr;
  double2* d_rho = nullptr;
  double* d_ek = nullptr;
  double* d_far = nullptr;
  double* d_weights = nullptr;
  SamplerRep* d_srep = nullptr;
  double* d_qtab = nullptr;
  bool injected = false;
  // MD
  MdChunk* d_chunks = nullptr;
  int nchunks = 0;
  int* d_chunk_rep_begin = nullptr;
  double *d_ke_partial = nullptr, *d_ke = nullptr, *d_T = nullptr, *d_lambda = nullptr,
         *d_xi = nullptr, *d_xold = nullptr, *d_vold = nullptr;
  bool pending_scale = false;
  // EAM device
  float4 *d_frho = nullptr, *d_rhor = nullptr, *d_z2r = nullptr;
  void* d_fp = nullptr;
  double *d_emb = nullptr, *d_epair = nullptr;
  float* d_host32 = nullptr;   // [3 n] staging of rbmd_force_compute_host_f32 (positions in, forces out)
  // topology device
  int *d_term_atom = nullptr, *d_tmult = nullptr, *d_sc_off = nullptr, *d_sc_id = nullptr, *d_row_off = nullptr,
      *d_row_idx = nullptr, *d_sp_off = nullptr, *d_sp_id = nullptr, *d_comp = nullptr;
  double *d_tk = nullptr, *d_ta = nullptr, *d_sc_fac = nullptr, *d_rows = nullptr, *d_eterm = nullptr,
         *d_esc = nullptr, *d_sp_wd = nullptr;
  float* d_sp_wf = nullptr;
  // water device
  int* d_hoh = nullptr;
  double *d_ebond = nullptr, *d_eangle = nullptr, *d_ewcoul = nullptr;
  // snapshot for step replay
  double *d_snap = nullptr;
  int* d_snap_img = nullptr;
  // host pinned
  uint32_t* h_status = nullptr;
  int* h_maxcount = nullptr;
  // streams
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaEvent_t ev_tail = nullptr;   // end of the k-space stream's work of a step (after the join)
  long long step_count = 0;
  long long* d_step = nullptr;   // step index of the k-samplers on the device (graph replay)
  long long* d_lstep = nullptr;  // Langevin noise counter (advanced after every application)
  double langevin_gamma = 100.0; // execution.langevin_gamma (the reference hard-codes 100)
  bool langevin_shared = false;  // compat.langevin_reference: m = 1, kBT = 1, one xi for all
  double langevin_xi[3] = {0, 0, 0};
  bool in_step = false;          // launches belong to rbmd_force_step (advance d_step)
  // the k-set of the next step was drawn at the end of the last step's k-space chain (own
  // samplers); any host-side change of sampler state clears it (drop_graphs)
  bool presampled = false;
  bool use_graph = true;         // execution.cuda_graph: replay a captured step
  cudaGraphExec_t graph_exec = nullptr;
  cudaGraphExec_t graph_multi = nullptr;   // graph_steps consecutive steps in one graph
  int graph_steps = 8;                     // execution.graph_steps
  int graph_multi_launches = 0;
  bool graph_multi_pending = false;
  int graph_launches = 0;
  bool graph_pending = false;    // pending_scale the graph was captured with
  bool capturing = false;
  cudaStream_t gstream = nullptr;
  cudaEvent_t ev_begin = nullptr;
  // captured steps put the cell sort and list build of a Verlet-skin step in a conditional graph
  // node (cond_rebuild); cstream captures its body.  Cleared for good when a capture with it fails.
  bool cond_rebuild = true;
  bool cond_failed = false;
  cudaStream_t cstream = nullptr;
  int launches = 0;
  // per-phase CUDA-event profiler (rbmd_force_profile / rbmd_force_phase_ms)
  bool prof_on = false;
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> prof_pairs;
  double phase_ms[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  long long phase_n[8] = {0, 0, 0, 0, 0, 0, 0, 0};

  bool is_rbe() const { return far && (coul_type == "RBE" || coul_type == "EWALD"); }
  bool is_rbl() const { return nbr_type == "RBL"; }
  bool is_eam() const { return ff == "EAM"; }
  bool is_cvff() const { return ff == "CVFF"; }
  bool with_coul_near() const { return far && ff != "EAM"; }
  double list_cut() const { return rc + skin; }
  // Verlet lists order cells by x (the RBL lists keep the reference's order by caller id)
  bool sort_x() const { return nbr_type != "RBL" && num_cycles == 1; }
};

namespace {

// phases: 0 integrate, 1 cell sort, 2 structure factors (side stream), 3 neighbour list,
// 4 near / EAM force pass, 5 constraints + intramolecular terms, 6 k sampler (side stream),
// 7 RBE force (side stream)
enum Phase {
  kPhInt = 0, kPhSort = 1, kPhK = 2, kPhList = 3, kPhForce = 4, kPhMol = 5, kPhSample = 6, kPhRbeF = 7
};

cudaEvent_t prof_event(rbmd_force* f) {
  if (f->ev_used == f->ev_pool.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    f->ev_pool.push_back(e);
  }
  return f->ev_pool[f->ev_used++];
}
struct PhaseScope {
  rbmd_force* f;
  int ph;
  cudaStream_t s;
  cudaEvent_t a = nullptr;
  PhaseScope(rbmd_force* f_, int ph_, cudaStream_t s_) : f(f_), ph(ph_), s(s_) {
    if (f->prof_on) {
      a = prof_event(f);
      cudaEventRecord(a, s);
    }
  }
  ~PhaseScope() {
    if (f->prof_on) {
      cudaEvent_t b = prof_event(f);
      cudaEventRecord(b, s);
      f->prof_pairs.push_back({ph, {a, b}});
    }
  }
};
// after the stream has been synchronised
void prof_collect(rbmd_force* f) {
  for (auto& p : f->prof_pairs) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, p.second.first, p.second.second) == cudaSuccess) {
      f->phase_ms[p.first] += ms;
      f->phase_n[p.first] += 1;
    }
  }
  f->prof_pairs.clear();
  f->ev_used = 0;
}

SpecialDev special_dev(const rbmd_force* f) {
  SpecialDev d;
  d.off = f->d_sp_off;
  d.id = f->d_sp_id;
  d.wf = f->d_sp_wf;
  d.wd = f->d_sp_wd;
  return d;
}

// LJ pair mode of the near passes: 0 none, 1 same-molecule exclusion, 2 special-bond weights.
int molecular_mode(const rbmd_force* f) {
  if (f->topo && f->special && f->is_cvff()) return 2;
  return f->at.molecule != nullptr ? 1 : 0;
}

// k_near_lean applies: one LJ coefficient pair for all types, no molecules, one thread per atom,
// no per-pair minimum image (a Verlet skin, or boxes of >= 3 cells per axis).
bool lean_ok(const rbmd_force* f) {
  return f->near_variant >= 1 && !f->is_rbl() && !f->is_eam() && f->nt_eff == 1 && molecular_mode(f) == 0 &&
         f->near_lanes == 1 && (f->skin > 0 || !f->minimg);
}

// The lean near pass and the per-atom list build run beside the k-space stream and use no shared
// memory, so an SM running them is configured for the largest L1; a k-space block that needs
// shared memory (staged atoms or k records, CDF tables, per-band sums) cannot start on such an SM
// until it drains, and the k-space chain then waited for the end of the near pass.  These two
// kernels therefore prefer half of the unified L1 as shared memory (their times are unchanged;
// the 1M-atom step 0.599 -> 0.585 ms), set once per device and kernel, outside stream capture.
// The lanes-per-atom and RBL passes of the small systems keep the default (the same preference
// slowed water by 5 % and the flexible chains by 3 %).
constexpr int kCallerCarveout = 50;
void prefer_shared_carveout(const rbmd_force* f, const void* fn) {
  if (!f->is_rbe() || f->capturing) return;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return;
  static std::mutex mu;
  static std::set<std::pair<int, const void*>> done;
  std::lock_guard<std::mutex> lock(mu);
  if (done.insert({dev, fn}).second)
    cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, kCallerCarveout);
}

void free_topology(rbmd_force* f) {
  dfree(f->d_term_atom); dfree(f->d_tmult); dfree(f->d_sc_off); dfree(f->d_sc_id); dfree(f->d_row_off);
  dfree(f->d_row_idx); dfree(f->d_sp_off); dfree(f->d_sp_id); dfree(f->d_comp); dfree(f->d_tk); dfree(f->d_ta);
  dfree(f->d_sc_fac); dfree(f->d_rows); dfree(f->d_eterm); dfree(f->d_esc); dfree(f->d_sp_wd); dfree(f->d_sp_wf);
}

void free_all(rbmd_force* f) {
  dfree(f->d_reps); dfree(f->d_ljt);
  dfree(f->d_rep_of); dfree(f->d_cell_of); dfree(f->d_cell_count); dfree(f->d_cell_start);
  dfree(f->d_cursor); dfree(f->d_tmp); dfree(f->d_slot_atom); dfree(f->d_atom_slot);
  if (f->d_pos4) cudaFree(f->d_pos4);
  f->d_pos4 = nullptr;
  if (f->d_frac) cudaFree(f->d_frac);
  f->d_frac = nullptr;
  dfree(f->d_meta); dfree(f->d_nbr); dfree(f->d_count); dfree(f->d_maxcount); dfree(f->d_status);
  dfree(f->d_count2); dfree(f->d_mean_partial); dfree(f->d_erf_tab);
  dfree(f->d_prep); dfree(f->d_cdf); dfree(f->d_wbin); dfree(f->d_pw); dfree(f->d_mlp); dfree(f->d_mlp_t); dfree(f->d_h);
  dfree(f->d_spec); dfree(f->d_spec_init);
  dfree(f->d_rebuild); dfree(f->d_block_sums); dfree(f->d_cell_rep); dfree(f->d_xref); dfree(f->d_nbuilds);
  dfree(f->d_segs);
  f->nsegs = 0;
  dfree(f->d_eslot); dfree(f->d_esum);
  if (f->d_krec) cudaFree(f->d_krec);
  f->d_krec = nullptr;
  dfree(f->d_kvec); dfree(f->d_krep); dfree(f->d_qidx); dfree(f->d_items); dfree(f->d_rhorep);
  if (f->d_partial) cudaFree(f->d_partial);
  f->d_partial = nullptr;
  dfree(f->d_rho); dfree(f->d_ek); dfree(f->d_far); dfree(f->d_weights); dfree(f->d_srep); dfree(f->d_qtab);
  dfree(f->d_chunks); dfree(f->d_chunk_rep_begin); dfree(f->d_ke_partial); dfree(f->d_ke);
  dfree(f->d_T); dfree(f->d_lambda); dfree(f->d_xi); dfree(f->d_xold); dfree(f->d_vold);
  dfree(f->d_frho); dfree(f->d_rhor); dfree(f->d_z2r);
  if (f->d_fp) cudaFree(f->d_fp);
  f->d_fp = nullptr;
  dfree(f->d_emb); dfree(f->d_epair); dfree(f->d_hoh); dfree(f->d_ebond); dfree(f->d_eangle); dfree(f->d_ewcoul);
  free_topology(f);
  dfree(f->d_host32);
  dfree(f->d_snap); dfree(f->d_snap_img); dfree(f->d_step); dfree(f->d_lstep);
  if (f->graph_exec) cudaGraphExecDestroy(f->graph_exec);
  f->graph_exec = nullptr;
  if (f->graph_multi) cudaGraphExecDestroy(f->graph_multi);
  f->graph_multi = nullptr;
  if (f->gstream) cudaStreamDestroy(f->gstream);
  f->gstream = nullptr;
  if (f->ev_begin) cudaEventDestroy(f->ev_begin);
  f->ev_begin = nullptr;
  if (f->h_status) cudaFreeHost(f->h_status);
  f->h_status = nullptr;
  if (f->h_maxcount) cudaFreeHost(f->h_maxcount);
  f->h_maxcount = nullptr;
  if (f->side) cudaStreamDestroy(f->side);
  f->side = nullptr;
  if (f->cstream) cudaStreamDestroy(f->cstream);
  f->cstream = nullptr;
  for (auto e : f->ev_pool) cudaEventDestroy(e);
  f->ev_pool.clear();
  f->ev_used = 0;
  f->prof_pairs.clear();
  if (f->ev_fork) cudaEventDestroy(f->ev_fork);
  if (f->ev_join) cudaEventDestroy(f->ev_join);
  if (f->ev_tail) cudaEventDestroy(f->ev_tail);
  f->ev_fork = f->ev_join = f->ev_tail = nullptr;
}

// Replica geometry: ContPointLocator::SetRange/SetCutOff/SetRs in the reference's float
// arithmetic (ContPointLocator.h:44-73) for FP32 mode, and the same formulas in double for FP64.
void setup_replica(const rbmd_box& b, double cut, double rs, bool fp64, RepDev& r, int& ncyc) {
  std::memset(&r, 0, sizeof r);
  const float rcf = (float)cut, rsf = (float)rs;
  ncyc = fp64 ? (int)std::ceil(cut / rs) : (int)std::ceil(rcf / rsf);
  for (int d = 0; d < 3; ++d) {
    r.lo_f[d] = (float)b.lo[d];
    r.hi_f[d] = (float)b.hi[d];
    const float span = r.hi_f[d] - r.lo_f[d];
    r.lo_d[d] = b.lo[d];
    r.hi_d[d] = b.hi[d];
    r.box_d[d] = b.hi[d] - b.lo[d];
    int dims = fp64 ? (int)(r.box_d[d] / (cut / (double)ncyc)) : (int)(span / (rcf / (float)ncyc));
    if (dims < 1) dims = 1;
    r.dims[d] = dims;
    r.box_f[d] = span;
    r.dx_f[d] = span / (float)dims;
    r.wrap_f[d] = r.dx_f[d] * (float)dims;
    r.dx_d[d] = r.box_d[d] / (double)dims;
    r.wrap_d[d] = r.dx_d[d] * (double)dims;
  }
  r.volume = r.box_d[0] * r.box_d[1] * r.box_d[2];
  r.ncell = r.dims[0] * r.dims[1] * r.dims[2];
}

// RBL list sizing of ExecutionMD::ComputeRBLNearForce / ComputeRBLLJForce / ComputeRBLEAMForce
// (rbmd/framework/run/ExecutionMD.cpp:467-486,577-589,724-736) for replica r in the run's Real:
// rho = N / (Lx Ly Lz); rs_num = round(1 + 0.05/rho - 0.05) * rho * ceil(4/3 pi rs^3) + 1 (the
// EAM variant has no rounding factor), rc_num likewise, pice = ceil(1 / (sample / (rc_num - rs_num))).
template <class Real>
void rbl_sizes_t(int64_t natoms, const Real* box, double rs, double rc, double sample, bool eam, int64_t* z) {
  const Real rho = (Real)natoms / (box[0] * box[1] * box[2]);
  const float pif = 3.14159265358979323846f;
  const Real rs_r = (Real)rs, rc_r = (Real)rc;
  int64_t coeff = 1;
  if (!eam) coeff = (int64_t)std::round((Real)(1.0 + (0.05 / (double)rho - 0.05)));
  const double cs = std::ceil(4.0 / 3.0 * (double)pif * (double)rs_r * (double)rs_r * (double)rs_r);
  const double cc = std::ceil(4.0 / 3.0 * (double)pif * (double)rc_r * (double)rc_r * (double)rc_r);
  const double rf = (double)(eam ? rho : (Real)coeff * rho);
  z[0] = (int64_t)(rf * cs + 1);
  z[1] = (int64_t)(rf * cc + 1);
  const Real rate = (Real)sample / (Real)(z[1] - z[0]);
  z[2] = (int64_t)std::ceil(1.0 / (double)rate);
}
void rbl_sizes(const rbmd_force* f, int r, int64_t* z) {
  const int64_t na = f->rep_off[r + 1] - f->rep_off[r];
  const rbmd_box& b = f->boxes[r];
  if (f->fp64) {
    const double box[3] = {b.hi[0] - b.lo[0], b.hi[1] - b.lo[1], b.hi[2] - b.lo[2]};
    rbl_sizes_t<double>(na, box, f->rs, f->rc, f->rbl_sample_num, f->is_eam(), z);
  } else {
    const float box[3] = {(float)b.hi[0] - (float)b.lo[0], (float)b.hi[1] - (float)b.lo[1],
                          (float)b.hi[2] - (float)b.lo[2]};
    rbl_sizes_t<float>(na, box, f->rs, f->rc, f->rbl_sample_num, f->is_eam(), z);
  }
}

// The reference's ERF table for the RBL Coulomb term (rbmd/framework/model/ERFTable.h, read by
// ExecStaticTable::TableGnearValue, rbmd/framework/staticTable/ExecStaticTable.h:96-135): entry k
// (bits 15..25 of the float distance) holds Gnear(alpha = 0.1, d_k) evaluated as the reference's
// ExecForceFunction::Gnear does in float ((1.0 - erf(x)) / d^2 in double, the rest in float,
// rbmd/framework/forceFunction/ExecForceFunction.h:217-224) at d_k = the bucket's lower edge
// rounded up to 4 decimals below d = 2 and to 3 decimals above, and not below 0.1, then rounded
// to the 6 significant decimal digits the reference's table literals carry.  Entries 921..2047
// cover 0.1 <= d < 2, entries 0..639 cover 2 <= d < 12; the rule reproduces 1734 of the 1766
// entries exactly and the other 32 to one unit in their sixth digit (at most 5e-6 relative).
std::vector<float> rbl_erf_table() {
  std::vector<float> t(2048, 0.f);
  auto fill = [&](int k0, int k1, int exp_base, int dec) {
    for (int k = k0; k < k1; ++k) {
      const int e3 = k >> 8, man = k & 255;
      const int ex = exp_base + (e3 >= 3 ? e3 - 3 : e3);
      const uint32_t bits = ((uint32_t)ex << 23) | ((uint32_t)man << 15);
      float edge;
      std::memcpy(&edge, &bits, 4);
      const double sc = std::pow(10.0, dec);
      const double v = (double)edge * sc, rv = std::nearbyint(v);
      double d = (std::fabs(v - rv) < 1e-6 ? rv : std::ceil(v)) / sc;
      d = std::max(d, 0.1);
      const float df = (float)d, a = 0.1f;
      const float x = std::sqrt(a) * df;
      const double t1 = (1.0 - (double)std::erf(x)) / (double)(df * df);
      const float pif = 3.14159265358979323846f;
      const float t2 = 2.0f * std::sqrt(a) * std::exp(-a * df * df) / (std::sqrt(pif) * df);
      char buf[32];
      std::snprintf(buf, sizeof buf, "%.6g", (double)(float)(t1 + (double)t2));
      t[k] = (float)std::strtod(buf, nullptr);
    }
  };
  fill(921, 2048, 123, 4);   // exponents 123..127 -> index high bits 3..7
  fill(0, 640, 128, 3);      // exponents 128..130 -> index high bits 0..2
  return t;
}

// Tables of the own k-proposal per replica: the 1D Gaussian g_d(m) = exp(-pi^2 m^2 / (alpha L_d^2))
// on |m| <= M_d with M_d = ceil(6 sqrt(alpha) L_d / pi) (so g_d(M_d) <= e^-36), its cumulative
// distribution (inverse-CDF sampling), and the mass W_b of p(m) = prod_d g_d(m_d) / (prod_d G_d - 1)
// (m != 0) in each |k| bin, accumulated over the octant |m_d| with multiplicities (the bin of m
// depends on |m_d| only).  Network parameters start at zero (h = 0: the Gaussian itself).
rbmd_status build_proposal_tables(rbmd_force* f, const std::vector<int64_t>& qoff) {
  const int nrep = f->nrep;
  f->prep_h.assign(nrep, PropRep{});
  f->wbin_h.assign((size_t)nrep * kPropBins, 0.0);
  std::vector<double> cdf;
  for (int r = 0; r < nrep; ++r) {
    PropRep& pr = f->prep_h[r];
    const double* L = f->reps_h[r].box_d;
    pr.kscale = 1.0 / (2.0 * std::sqrt(f->alpha));
    pr.nq = (int)(qoff[r + 1] - qoff[r]);
    std::vector<double> g[3];
    double G[3];
    for (int d = 0; d < 3; ++d) {
      pr.c[d] = 2.0 * M_PI / L[d];
      pr.M[d] = (int)std::ceil(6.0 * std::sqrt(f->alpha) * L[d] / M_PI);
      if (pr.M[d] > (1 << 16)) {
        std::snprintf(g_last_error, sizeof g_last_error, "proposal: box too large for the k tables");
        return RBMD_ERR_CONFIG;
      }
      const double c = M_PI * M_PI / (f->alpha * L[d] * L[d]);
      g[d].resize(pr.M[d] + 1);
      for (int m = 0; m <= pr.M[d]; ++m) g[d][m] = std::exp(-c * (double)m * (double)m);
      G[d] = g[d][0];
      for (int m = 1; m <= pr.M[d]; ++m) G[d] += 2.0 * g[d][m];
      pr.cdf_off[d] = (int)cdf.size();
      double acc = 0;
      for (int m = -pr.M[d]; m <= pr.M[d]; ++m) {
        acc += g[d][std::abs(m)];
        cdf.push_back(acc / G[d]);
      }
      cdf.back() = 1.0;
    }
    const double Z = G[0] * G[1] * G[2] - 1.0;
    double* W = f->wbin_h.data() + (size_t)r * kPropBins;
    for (int a = 0; a <= pr.M[0]; ++a)
      for (int b = 0; b <= pr.M[1]; ++b) {
        const double gab = g[0][a] * g[1][b] * (a ? 2.0 : 1.0) * (b ? 2.0 : 1.0);
        for (int c = 0; c <= pr.M[2]; ++c) {
          if (a == 0 && b == 0 && c == 0) continue;
          W[prop_bin(prop_kappa(pr, a, b, c))] += gab * g[2][c] * (c ? 2.0 : 1.0);
        }
      }
    for (int k = 0; k < kPropBins; ++k) W[k] /= Z;
  }
  f->prop_stage_bytes = 0;
  for (const PropRep& pr : f->prep_h)
    f->prop_stage_bytes = std::max(f->prop_stage_bytes, (int)sizeof(double) * prop_stage_doubles(pr));
  CK(dalloc(&f->d_prep, (size_t)nrep));
  CK(cudaMemcpy(f->d_prep, f->prep_h.data(), sizeof(PropRep) * nrep, cudaMemcpyHostToDevice));
  CK(dalloc(&f->d_cdf, cdf.size()));
  CK(cudaMemcpy(f->d_cdf, cdf.data(), sizeof(double) * cdf.size(), cudaMemcpyHostToDevice));
  CK(dalloc(&f->d_wbin, f->wbin_h.size()));
  CK(cudaMemcpy(f->d_wbin, f->wbin_h.data(), sizeof(double) * f->wbin_h.size(), cudaMemcpyHostToDevice));
  CK(dalloc(&f->d_pw, (size_t)f->Ptot));
  CK(dalloc(&f->d_mlp, (size_t)kMlpNParam));
  CK(dalloc(&f->d_mlp_t, (size_t)kMlpNParam));
  CK(cudaMemset(f->d_mlp, 0, sizeof(float) * kMlpNParam));
  CK(dalloc(&f->d_h, (size_t)nrep * kPropBins));
  CK(dalloc(&f->d_spec, (size_t)nrep * kPropBands));
  CK(cudaMemset(f->d_spec, 0, sizeof(float) * nrep * kPropBands));
  CK(dalloc(&f->d_spec_init, (size_t)nrep));
  CK(cudaMemset(f->d_spec_init, 0, sizeof(int) * nrep));
  f->prop_trained = false;
  return RBMD_OK;
}

// Scratch of one training run, freed on every return path.
struct TrainScratch {
  std::vector<void*> ptrs;
  template <class T>
  cudaError_t get(T** p, size_t count) {
    cudaError_t e = dalloc(p, count);
    if (e == cudaSuccess) ptrs.push_back((void*)*p);
    return e;
  }
  ~TrainScratch() {
    for (void* p : ptrs) cudaFree(p);
  }
};

// Fit of the proposal network to S snapshots (cbin, spec on the device): inputs from each
// snapshot's spectrum, W_b of replica 0, parameters initialised with an output layer of zero
// (h = 0, the Gaussian, at the start), full-batch Adam with a cosine-decayed learning rate
// (floor 0.1), mean group loss reported before, at the first step and after the last; the
// network's conditioning state starts at the mean training spectrum.
rbmd_status train_fit(rbmd_force* f, const rbmd_train_opts* o, rbmd_train_report* rep, cudaStream_t s,
                      std::chrono::steady_clock::time_point t0, int S, float* cbin, float* spec, float* wbinf,
                      float* X, double* loss, float* gpart, float* grad, float* am, float* av) {
  std::vector<float> wf((size_t)S * kPropBins);
  for (int sn = 0; sn < S; ++sn)
    for (int b = 0; b < kPropBins; ++b) wf[(size_t)sn * kPropBins + b] = (float)f->wbin_h[b];
  CK(cudaMemcpyAsync(wbinf, wf.data(), sizeof(float) * wf.size(), cudaMemcpyHostToDevice, s));
  k_prop_features<<<(S * kPropBins + 255) / 256, 256, 0, s>>>(S, spec, X);
  std::vector<float> p(kMlpNParam, 0.f);
  {
    std::mt19937_64 rng(o->seed * 0x9E3779B97F4A7C15ull + 17);
    std::normal_distribution<float> nd(0.f, 1.f);
    for (int e = 0; e < kMlpHid * kMlpIn; ++e) p[kOW1 + e] = nd(rng) / 4.0f;
    for (int e = 0; e < kMlpHid * kMlpHid; ++e) p[kOW2 + e] = nd(rng) / 8.0f;
    for (int j = 0; j < kMlpHid; ++j) {
      p[kOB1 + j] = 0.1f * nd(rng);
      p[kOB2 + j] = 0.1f * nd(rng);
    }
  }
  CK(cudaMemcpyAsync(f->d_mlp, p.data(), sizeof(float) * kMlpNParam, cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(am, 0, sizeof(float) * kMlpNParam, s));
  CK(cudaMemsetAsync(av, 0, sizeof(float) * kMlpNParam, s));
  MlpArgs a{};
  a.groups = S;
  a.train = 1;
  a.gscale = 1.0f / (float)S;
  a.params = f->d_mlp;
  a.x = X;
  a.wbin = wbinf;
  a.cbin = cbin;
  a.h = nullptr;
  a.loss = loss;
  a.grad_partial = gpart;
  a.status = f->d_status;
  std::vector<double> lh(S);
  auto mean_loss = [&]() -> double {
    cudaMemcpyAsync(lh.data(), loss, sizeof(double) * S, cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    double m = 0;
    for (double v : lh) m += v;
    return m / S;
  };
  const int T = o->iterations;
  double l_first = 0;
  for (int it = 1; it <= T; ++it) {
    CK(mlp_launch(a, s));
    CK(mlp_grad_sum(S, gpart, grad, s));
    const float lr = o->learning_rate * (0.1f + 0.45f * (1.0f + std::cos((float)M_PI * (float)(it - 1) / (float)T)));
    CK(mlp_adam(f->d_mlp, grad, am, av, lr, it, s));
    if (it == 1) l_first = mean_loss();
  }
  CK(mlp_launch(a, s));
  const double l_final = mean_loss();
  uint32_t st = 0;
  CK(cudaMemcpy(&st, f->d_status, sizeof st, cudaMemcpyDeviceToHost));
  if (st & kFlagMlpTimeout) {
    std::snprintf(g_last_error, sizeof g_last_error, "train_proposal: a tensor-core wait timed out");
    return RBMD_ERR_DEVICE;
  }
  // reference losses from the data: h = 0 (Gaussian) and the per-snapshot optimum
  std::vector<float> cb((size_t)S * kPropBins), sp((size_t)S * kPropBands);
  CK(cudaMemcpy(cb.data(), cbin, sizeof(float) * cb.size(), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(sp.data(), spec, sizeof(float) * sp.size(), cudaMemcpyDeviceToHost));
  double lg = 0, lo = 0;
  for (int sn = 0; sn < S; ++sn) {
    double sw = 0, sc = 0, sq = 0;
    for (int b = 0; b < kPropBins; ++b) {
      const double w = f->wbin_h[b], c = cb[(size_t)sn * kPropBins + b];
      sw += w;
      sc += c;
      sq += std::sqrt(w * c);
    }
    lg += std::log(sw) + std::log(sc);
    lo += 2.0 * std::log(sq);
  }
  lg /= S;
  lo /= S;
  std::vector<float> mean_spec(kPropBands, 0.f);
  for (int sn = 0; sn < S; ++sn)
    for (int j = 0; j < kPropBands; ++j) mean_spec[j] += sp[(size_t)sn * kPropBands + j] / (float)S;
  std::vector<float> spec_all((size_t)f->nrep * kPropBands);
  for (int r = 0; r < f->nrep; ++r)
    for (int j = 0; j < kPropBands; ++j) spec_all[(size_t)r * kPropBands + j] = mean_spec[j];
  CK(cudaMemcpy(f->d_spec, spec_all.data(), sizeof(float) * spec_all.size(), cudaMemcpyHostToDevice));
  std::vector<int> ones(f->nrep, 1);
  CK(cudaMemcpy(f->d_spec_init, ones.data(), sizeof(int) * f->nrep, cudaMemcpyHostToDevice));
  CK(mlp_prepare(f->d_mlp, f->d_mlp_t, s));
  f->prop_trained = true;
  f->presampled = false;
  if (rep) {
    rep->loss_gauss = lg;
    rep->loss_first = l_first;
    rep->loss_final = l_final;
    rep->loss_optimum = lo;
    rep->variance_ratio = std::exp(l_final - lg);
    rep->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  return RBMD_OK;
}

// RBE normaliser S = prod_d H_d - 1 with H_d = sqrt(a L^2/pi) sum_{|m|<=10} e^{-a L^2 m^2}
// (ExecForceFunction::Compute_S/Compute_H, rbmd/framework/forceFunction/ExecForceFunction.h:266-294),
// evaluated in FP64.
double rbe_S(double alpha, const double* L) {
  double H[3];
  for (int i = 0; i < 3; ++i) {
    const double factor = -(alpha * L[i] * L[i]);
    double h = 0;
    for (int m = -10; m <= 10; ++m) h += std::exp((double)(m * m) * factor);
    H[i] = h * std::sqrt(-factor / M_PI);
  }
  return H[0] * H[1] * H[2] - 1.0;
}

template <class R>
void launch_nlist(rbmd_force* f, cudaStream_t s) {
  PhaseScope ps(f, kPhList, s);
  if (f->tpa_list == 0 && f->nsegs > 0) {
    const size_t smem = (size_t)f->stage_cap * sizeof(typename Traits<R>::V4);
    k_nlist_staged<R><<<f->nsegs, kStageThreads, smem, s>>>(
        f->d_segs, f->stage_cap, (const typename Traits<R>::V4*)f->d_pos4, f->d_cell_start, f->d_reps,
        (R)f->list_cut(), f->cap, f->stride, f->d_nbr, f->d_count, f->d_maxcount, f->d_status,
        f->skin > 0 ? f->d_rebuild : nullptr, f->d_nbuilds, f->sort_x() ? 1 : 0, f->nrep, f->orig_pred ? 1 : 0);
    f->launches++;
    return;
  }
  if (f->tpa_list == 1 && f->num_cycles == 1) {   // warp per atom
    k_nlist_warp<R><<<(f->n + 7) / 8, 256, 0, s>>>(
        f->n, (const typename Traits<R>::V4*)f->d_pos4, f->d_cell_start, f->d_reps,
        f->nrep > 1 ? f->d_rep_of : nullptr, (R)f->list_cut(), f->cap, f->stride, f->d_nbr, f->d_count,
        f->d_maxcount, f->d_status, f->skin > 0 ? f->d_rebuild : nullptr, f->d_nbuilds, f->nrep,
        f->orig_pred ? 1 : 0);
    f->launches++;
    return;
  }
  const int bs = f->tpa_list > 1 ? f->tpa_list : 128;
  prefer_shared_carveout(f, (const void*)k_nlist<R>);
  k_nlist<R><<<(f->n + bs - 1) / bs, bs, 0, s>>>(
      f->n, (const typename Traits<R>::V4*)f->d_pos4, f->d_cell_start, f->d_reps,
      f->nrep > 1 ? f->d_rep_of : nullptr, f->num_cycles, (R)f->list_cut(), f->cap, f->stride, f->d_nbr,
      f->d_count, f->d_maxcount, f->d_status, f->skin > 0 ? f->d_rebuild : nullptr, f->d_nbuilds,
      f->sort_x() ? 1 : 0, f->nrep, f->orig_pred ? 1 : 0);
  f->launches++;
}

template <class R>
void launch_rbl_list(rbmd_force* f, cudaStream_t s) {
  PhaseScope ps(f, kPhList, s);
  const int* rp = f->nrep > 1 ? f->d_rep_of : nullptr;
  const int side = 2 * f->num_cycles + 1;
  // one warp per atom below 10 warps' worth of atoms per SM (measured crossover between 21k and
  // 98k atoms on B200), where one thread per atom leaves most SMs idle
  const bool warp = f->rbl_list_warp > 0 || (f->rbl_list_warp < 0 && f->n < 10 * 32 * f->num_sms);
  if (warp && side * side * side <= kRblStencilMax) {
    k_rbl_list_warp<R><<<(f->n + kRblWarps - 1) / kRblWarps, 32 * kRblWarps, 0, s>>>(
        f->n, (const typename Traits<R>::V4*)f->d_pos4, f->d_cell_start, f->d_reps, rp, f->num_cycles, (R)f->rc,
        (R)f->rs, f->core_cap, f->shell_cap, f->stride, f->d_nbr, f->d_count, f->d_count2, f->d_maxcount,
        f->d_status);
  } else {
    k_rbl_list<R><<<(f->n + 127) / 128, 128, 0, s>>>(
        f->n, (const typename Traits<R>::V4*)f->d_pos4, f->d_cell_start, f->d_reps, rp, f->num_cycles, (R)f->rc,
        (R)f->rs, f->core_cap, f->shell_cap, f->stride, f->d_nbr, f->d_count, f->d_count2, f->d_maxcount,
        f->d_status);
  }
  f->launches++;
}

// List reuse under a Verlet skin: refresh the slot caches of the replicas that keep their list
// from the new positions (the cell sort refreshes the others).
template <class R>
void launch_regather(rbmd_force* f, cudaStream_t s) {
  const int n = f->n;
  k_regather<R><<<(n + 255) / 256, 256, 0, s>>>(
      n, f->d_slot_atom, f->at.pos, f->at.charge, f->nrep > 1 ? f->d_rep_of : nullptr, f->d_reps,
      (typename Traits<R>::V4*)f->d_pos4, nullptr, f->d_xref, f->d_rebuild);
  f->launches++;
}

// bin: run k_bin (positions given by the caller, or a Verlet skin whose drift does not bin);
// regather: refresh the slot caches on list-reuse steps (the drift did not write them).
template <class R>
void launch_sort(rbmd_force* f, cudaStream_t s, bool bin, bool regather) {
  PhaseScope ps(f, kPhSort, s);
  const int n = f->n;
  // per-replica rebuild flags (Verlet skin): rb[r], and rb[nrep] = any replica
  const int* rb = f->skin > 0 ? f->d_rebuild : nullptr;
  const int* rb_any = rb ? rb + f->nrep : nullptr;
  const int* rep_of = f->nrep > 1 ? f->d_rep_of : nullptr;
  if (bin) {
    if (rb) {
      k_zero_counts<<<(f->ncell_total + 255) / 256, 256, 0, s>>>(f->ncell_total, f->d_cell_rep, rb,
                                                                  f->d_cell_count);
      f->launches++;
    } else {
      cudaMemsetAsync(f->d_cell_count, 0, sizeof(int) * f->ncell_total, s);
    }
    k_bin<R><<<(n + 255) / 256, 256, 0, s>>>(n, f->at.pos, rep_of, f->d_reps, f->d_cell_of, f->d_cell_count,
                                             f->d_status, rb);
    f->launches++;
  }
  const int nblk = (f->ncell_total + kScanBlock - 1) / kScanBlock;
  k_cell_block_sums<<<nblk, 1024, 0, s>>>(f->ncell_total, f->d_cell_count, f->d_block_sums, rb_any,
                                          f->d_status);
  k_cell_scan<<<nblk, 1024, 0, s>>>(f->ncell_total, f->d_cell_count, f->d_block_sums, f->d_cell_start,
                                    f->d_cursor, rb_any);
  k_scatter<<<(n + 255) / 256, 256, 0, s>>>(n, f->d_cell_of, f->d_cell_start, f->d_cursor, f->d_tmp, rep_of,
                                            rb);
  k_cell_sort_gather<R><<<(f->ncell_total + kSortWarps - 1) / kSortWarps, 32 * kSortWarps, 0, s>>>(
      f->ncell_total, f->d_cell_start, f->d_tmp, f->at.pos, f->at.charge, f->at.type,
      molecular_mode(f) == 2 ? f->d_comp : f->at.molecule,
      rep_of, f->d_reps, f->d_slot_atom, f->d_atom_slot, (typename Traits<R>::V4*)f->d_pos4, nullptr,
      f->d_meta, f->d_xref, rb, f->sort_x() ? 1 : 0, f->d_cell_rep);
  f->launches += 4;
  if (rb && regather) launch_regather<R>(f, s);
}

// Samples of the own proposal for `step`: with a trained network the per-bin log-weights h come
// from the network evaluated on the current conditioning spectrum (tensor cores), then the exact
// sampler draws from q = p e^h / Z with weights p / q; otherwise it draws from p.
void launch_prop_sample(rbmd_force* f, cudaStream_t s, long long step, int rec_bytes,
                        const long long* step_dev = nullptr) {
  const float* h = nullptr;
  if (f->proposal == "learned" && f->prop_trained) {
    k_prop_h<<<(kMlpLanes * f->nrep * kPropBins + 255) / 256, 256, 0, s>>>(f->nrep, f->d_mlp_t, f->d_spec, f->d_h);
    h = f->d_h;
    f->launches++;
  }
  k_prop_sample<<<f->nrep, kSampThreads, f->prop_stage_bytes, s>>>(f->nrep, f->d_reps, f->d_prep, f->d_cdf, h, f->d_wbin, f->seed,
                                                 step, step_dev, 4096, f->d_kvec, f->d_krec, rec_bytes, f->d_krep,
                                                 f->d_pw, f->d_status);
  f->launches++;
}

// k-space chain on the side stream: sampler (depends only on the step counter, so it runs
// before the fork wait), fixed-point fractional coordinates, structure factors, coefficients,
// RBE force into d_far.
template <class R>
void launch_kspace(rbmd_force* f, cudaStream_t s, cudaEvent_t ready) {
  const int rec_bytes = sizeof(typename KRec<R>::T);
  if (f->capturing) cudaStreamWaitEvent(s, f->ev_begin, 0);   // the side stream joins the capture
  const bool own = !f->injected && f->coul_type == "RBE";
  const bool own_prop = own && f->proposal != "gauss";
  // the own sampler for the step index in the device counter
  auto sample = [&] {
    PhaseScope ps(f, kPhSample, s);
    if (!own_prop) {
      k_sample<kSamplerD><<<f->nrep, 256, 0, s>>>(f->nrep, f->d_srep, f->d_qtab, f->d_reps, f->seed,
                                                  f->step_count, f->d_step, f->d_kvec, f->d_krec, rec_bytes,
                                                  f->d_krep, f->d_status);
      f->launches++;
    } else {
      launch_prop_sample(f, s, f->step_count, rec_bytes, f->d_step);
    }
  };
  // this step's k-set, unless the last step's chain drew it already
  if (own && !f->presampled) sample();
  f->presampled = false;
  cudaStreamWaitEvent(s, ready, 0);
  if (f->nq == 0) {
    cudaEventRecord(f->ev_join, s);
    if (f->in_step) {
      k_step_inc<<<1, 1, 0, s>>>(f->d_step);
      f->launches++;
    }
    cudaEventRecord(f->ev_tail, s);
    return;
  }
  const int* rep_of = f->nrep > 1 ? f->d_rep_of : nullptr;
  {
    PhaseScope ps(f, kPhK, s);
    k_frac<R><<<(f->nq + 255) / 256, 256, 0, s>>>(f->nq, f->d_qidx, f->at.pos, f->at.charge, rep_of,
                                                   f->d_reps, f->d_frac);
    k_rho_lanes<R, kKL><<<f->nitems, f->rho_threads, 0, s>>>(
        f->d_items, (const typename FracT<R>::T*)f->d_frac, (const typename KRec<R>::T*)f->d_krec,
        (R*)f->d_partial, f->ktile);
    k_rho_finish<R><<<(f->Ptot + 3) / 4, 128, 0, s>>>(
        f->Ptot, f->ktile, f->d_krep, f->d_rhorep, f->d_reps, (const R*)f->d_partial,
        own_prop ? f->d_pw : f->d_weights, f->u.qqr2e, (typename KRec<R>::T*)f->d_krec, f->d_rho, f->d_ek);
  }
  {
    PhaseScope ps(f, kPhRbeF, s);
    const size_t smem = (size_t)f->kstage * sizeof(typename KRec<R>::T);
    k_rbe_force<R><<<(f->nq + 127) / 128, 128, smem, s>>>(
        f->nq, f->kstage, f->d_qidx, (const typename FracT<R>::T*)f->d_frac,
        (const typename KRec<R>::T*)f->d_krec, f->d_reps, rep_of, f->d_far);
  }
  f->launches += 4;
  // conditioning of the next step's proposal, after the force kernels of this one
  if (own_prop && f->proposal == "learned" && f->prop_trained) {
    k_prop_spectrum<<<f->nrep, 256, 0, s>>>(f->nrep, f->d_reps, f->d_prep, f->d_kvec, f->d_rho, f->d_pw, 0.1f,
                                            f->d_spec, f->d_spec_init);
    f->launches++;
  }
  // the caller stream joins here (ev_join): the step counter and the next step's k-set come after
  cudaEventRecord(f->ev_join, s);
  if (f->in_step) {
    k_step_inc<<<1, 1, 0, s>>>(f->d_step);
    f->launches++;
    // the next step's k-set, drawn behind the join: the sampler depends only on the step counter
    // and the conditioning spectrum just updated, so it overlaps the caller's kick, thermostat and
    // next drift instead of opening the next step's chain ahead of its structure factors
    if (own) {
      sample();
      f->presampled = true;
    }
  }
  cudaEventRecord(f->ev_tail, s);
}

template <class R, bool COUL, int MI>
void launch_near_t(rbmd_force* f, cudaStream_t s) {
  NearParams p;
  p.n = f->n;
  p.stride = f->stride;
  p.ntypes = f->nt_eff;
  p.cap = f->cap;
  p.with_lj = 1;
  p.with_coul = COUL;
  p.molecular = molecular_mode(f);
  p.sp = special_dev(f);
  p.rc = f->rc;
  p.alpha = f->alpha;
  p.coul_scale = f->near_coul_scale;
  p.sqrt_alpha = std::sqrt(f->alpha);
  p.two_sqrt_alpha_over_sqrt_pi = 2.0 * std::sqrt(f->alpha) / std::sqrt(M_PI);
  p.kstage = 0;
  p.orig = f->orig_pred ? 1 : 0;
  if (f->near_lanes > 1) {
    const long long threads = (long long)f->n * f->near_lanes;
    const int grid = (int)((threads + 255) / 256);
    auto kern = f->near_lanes == 4    ? k_near_force_group<R, COUL, MI, 4>
                : f->near_lanes == 8  ? k_near_force_group<R, COUL, MI, 8>
                : f->near_lanes == 16 ? k_near_force_group<R, COUL, MI, 16>
                                      : k_near_force_group<R, COUL, MI, 32>;
    kern<<<grid, 256, 0, s>>>(p, f->d_ljt, (const typename Traits<R>::V4*)f->d_pos4, f->d_meta, f->d_nbr,
                              f->d_count, f->d_reps, f->nrep > 1 ? f->d_rep_of : nullptr, f->d_slot_atom,
                              f->at.force, f->want_energy ? f->d_eslot : nullptr, f->d_status);
    f->launches++;
    return;
  }
  const int bs = f->tpa_near;
  if constexpr ((MI & 3) != kMiLJ && (MI & kMiSpecial) == 0) {
    // one LJ coefficient pair for all types, no molecules: the lean pass
    if (lean_ok(f)) {
      auto kern = f->want_energy ? k_near_lean<R, COUL, MI, true> : k_near_lean<R, COUL, MI, false>;
      prefer_shared_carveout(f, (const void*)kern);
      kern<<<(f->n + bs - 1) / bs, bs, 0, s>>>(
          p, lj24<R>(f->ljt_h, 0), sig6<R>(f->ljt_h, 0), (const typename Traits<R>::V4*)f->d_pos4, f->d_nbr,
          f->d_count, f->d_reps, f->nrep > 1 ? f->d_rep_of : nullptr, f->d_slot_atom, f->at.force,
          f->want_energy ? f->d_eslot : nullptr, f->d_status);
      f->launches++;
      return;
    }
  }
  k_near_force<R, COUL, MI><<<(f->n + bs - 1) / bs, bs, 0, s>>>(
      p, f->d_ljt, (const typename Traits<R>::V4*)f->d_pos4, f->d_meta, f->d_nbr, f->d_count,
      f->d_reps, f->nrep > 1 ? f->d_rep_of : nullptr, f->d_slot_atom, f->at.force,
      f->want_energy ? f->d_eslot : nullptr, f->d_status);
  f->launches++;
}

template <class R, bool COUL>
void launch_near_m(rbmd_force* f, cudaStream_t s) {
  const int mi = f->skin > 0 ? kMiAll : (f->minimg ? kMiLJ : kMiNone);
  if (molecular_mode(f) == 2) {   // special-bond LJ weights: their own instantiations
    if (mi == kMiAll) launch_near_t<R, COUL, kMiAll | kMiSpecial>(f, s);
    else if (mi == kMiLJ) launch_near_t<R, COUL, kMiLJ | kMiSpecial>(f, s);
    else launch_near_t<R, COUL, kMiNone | kMiSpecial>(f, s);
    return;
  }
  if (mi == kMiAll) launch_near_t<R, COUL, kMiAll>(f, s);
  else if (mi == kMiLJ) launch_near_t<R, COUL, kMiLJ>(f, s);
  else launch_near_t<R, COUL, kMiNone>(f, s);
}

template <class R>
void launch_near(rbmd_force* f, cudaStream_t s) {
  if (f->with_coul_near()) launch_near_m<R, true>(f, s);
  else launch_near_m<R, false>(f, s);
}

template <class R>
void launch_eam(rbmd_force* f, cudaStream_t s) {
  EamDev e;
  e.frho = f->d_frho;
  e.rhor = f->d_rhor;
  e.z2r = f->d_z2r;
  e.nrho = f->eam_h.nrho;
  e.nr = f->eam_h.nr;
  e.rdr = 1.0f / f->eam_h.dr;
  e.rdrho = 1.0f / f->eam_h.drho;
  e.rdr_d = 1.0 / (double)f->eam_h.dr;
  e.rdrho_d = 1.0 / (double)f->eam_h.drho;
  e.rhomax = f->eam_h.rhomax;
  const int* rp = f->nrep > 1 ? f->d_rep_of : nullptr;
  const int bs = 128;
  const int nb = (f->n + bs - 1) / bs;
  auto fp_kern = f->minimg ? k_eam_fp<R, true> : k_eam_fp<R, false>;
  auto force_kern = f->minimg ? k_eam_force<R, true> : k_eam_force<R, false>;
  fp_kern<<<nb, bs, 0, s>>>(f->n, f->stride, f->cap, f->rc, e, (const typename Traits<R>::V4*)f->d_pos4,
                            f->d_nbr, f->d_count, f->d_reps, rp, (R*)f->d_fp, f->d_emb);
  force_kern<<<nb, bs, 0, s>>>(f->n, f->stride, f->cap, f->rc, e, (const typename Traits<R>::V4*)f->d_pos4,
                               f->d_nbr, f->d_count, f->d_reps, rp, (const R*)f->d_fp, f->d_slot_atom,
                               f->at.force, f->d_epair, f->d_status, f->eam_ref_sign ? 1 : 0);
  f->launches += 2;
}

// Lanes per atom of the RBL force pass: tuning.rbl_lanes, else 16 below 10 warps' worth of atoms
// per SM and 8 above (B200, flexible chains at rc 12 A with ~80 RBL entries per atom: 4k atoms
// 0.191 -> 0.034 ms, 21k 0.198 -> 0.064 ms, 50k 0.217 -> 0.122 ms, 98k 0.253 -> 0.200 ms against
// one thread per atom).
int rbl_lanes(const rbmd_force* f) {
  if (f->rbl_lanes > 0) return f->rbl_lanes;
  return f->n < 10 * 32 * f->num_sms ? 16 : 8;
}

template <class R, bool C, bool SP>
auto pick_rbl_force_g(int g) -> decltype(&k_rbl_force<R, C, SP, 1>) {
  switch (g) {
    case 4: return k_rbl_force<R, C, SP, 4>;
    case 8: return k_rbl_force<R, C, SP, 8>;
    case 16: return k_rbl_force<R, C, SP, 16>;
    case 32: return k_rbl_force<R, C, SP, 32>;
    default: return k_rbl_force<R, C, SP, 1>;
  }
}

template <class R>
auto pick_rbl_force(bool coul, bool spw, int g) -> decltype(&k_rbl_force<R, true, true, 1>) {
  if (coul) return spw ? pick_rbl_force_g<R, true, true>(g) : pick_rbl_force_g<R, true, false>(g);
  return spw ? pick_rbl_force_g<R, false, true>(g) : pick_rbl_force_g<R, false, false>(g);
}

template <class R>
void launch_rbl_force(rbmd_force* f, cudaStream_t s) {
  const int* rp = f->nrep > 1 ? f->d_rep_of : nullptr;
  const int nb = (f->n + 127) / 128;
  if (f->is_eam()) {
    EamDev e;
    e.frho = f->d_frho;
    e.rhor = f->d_rhor;
    e.z2r = f->d_z2r;
    e.nrho = f->eam_h.nrho;
    e.nr = f->eam_h.nr;
    e.rdr = 1.0f / f->eam_h.dr;
    e.rdrho = 1.0f / f->eam_h.drho;
    e.rdr_d = 1.0 / (double)f->eam_h.dr;
    e.rdrho_d = 1.0 / (double)f->eam_h.drho;
    e.rhomax = f->eam_h.rhomax;
    k_rbl_eam_fp<R><<<nb, 128, 0, s>>>(f->n, f->stride, f->core_cap, f->shell_cap, f->rc, f->rs, e,
                                        (const typename Traits<R>::V4*)f->d_pos4, f->d_nbr, f->d_count,
                                        f->d_count2, f->d_reps, rp, (R*)f->d_fp, f->d_emb);
    k_rbl_eam_force<R><<<nb, 128, 0, s>>>(f->n, f->stride, f->core_cap, f->shell_cap, f->rc, f->rs, e,
                                           (const typename Traits<R>::V4*)f->d_pos4, f->d_nbr, f->d_count,
                                           f->d_count2, f->d_reps, rp, (const R*)f->d_fp, f->d_slot_atom,
                                           f->at.force, f->d_epair, f->d_status);
    f->launches += 2;
  } else {
    RblParams p;
    p.n = f->n;
    p.stride = f->stride;
    p.ntypes = f->nt_eff;
    p.core_cap = f->core_cap;
    p.molecular = molecular_mode(f);
    p.sp = special_dev(f);
    p.table_mode = f->rbl_table ? 1 : 0;
    p.shell_coul = f->rbl_shell_coul ? 1 : 0;
    p.erf_tab = f->d_erf_tab;
    p.rc = f->rc;
    p.rs = f->rs;
    p.alpha = f->alpha;
    p.qqr2e = f->u.qqr2e;
    p.sqrt_alpha = std::sqrt(f->alpha);
    p.two_sqrt_alpha_over_sqrt_pi = 2.0 * std::sqrt(f->alpha) / std::sqrt(M_PI);
    double* es = f->want_energy ? f->d_eslot : nullptr;
    const bool spw = p.molecular == 2;
    const int g = rbl_lanes(f);
    auto kern = pick_rbl_force<R>(f->with_coul_near(), spw, g);
    const int grid = (int)(((long long)f->n * g + 127) / 128);
    kern<<<grid, 128, 0, s>>>(p, f->d_ljt, (const typename Traits<R>::V4*)f->d_pos4, f->d_meta, f->d_nbr,
                              f->d_count, f->d_count2, f->d_reps, rp, f->d_slot_atom, f->shell_cap, f->at.force, es,
                              f->d_status);
    f->launches++;
  }
  // F_i -= mean_j F_j per replica (ExecutionMD.cpp:568-570)
  k_force_chunk_sum<<<f->nchunks, 256, 0, s>>>(f->d_chunks, f->at.force, f->d_mean_partial);
  k_force_sub_mean<<<f->nchunks, 256, 0, s>>>(f->d_chunks, f->d_chunk_rep_begin, f->d_reps, f->d_mean_partial,
                                              f->at.force);
  f->launches += 2;
}

// float <-> double copies of the host-buffer call in the reference's own Vec3f layout.
__global__ void k_f32_to_f64(long long m, const float* __restrict__ a, double* __restrict__ b) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < m; k += (long long)gridDim.x * blockDim.x)
    b[k] = (double)a[k];
}
__global__ void k_f64_to_f32(long long m, const double* __restrict__ a, float* __restrict__ b) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < m; k += (long long)gridDim.x * blockDim.x)
    b[k] = (float)a[k];
}

// General topology: per-term forces, then the per-atom gather with the Coulomb correction.
void launch_bonded(rbmd_force* f, cudaStream_t s) {
  BondedParams bp;
  bp.n = f->n;
  bp.nb = f->topo_nb;
  bp.na = f->topo_na;
  bp.nd = f->topo_nd;
  bp.coul_const = 332.06371;
  const int* rep_of = f->nrep > 1 ? f->d_rep_of : nullptr;
  const int nterm = bp.nb + bp.na + bp.nd;
  if (nterm > 0) {
    k_bonded_terms<<<(nterm + 255) / 256, 256, 0, s>>>(bp, f->d_term_atom, f->d_tk, f->d_ta, f->d_tmult, f->at.pos,
                                                       rep_of, f->d_reps, f->d_rows, f->d_eterm);
    f->launches++;
  }
  k_bonded_gather<<<(f->n + 255) / 256, 256, 0, s>>>(bp, f->d_sc_off, f->d_sc_id, f->d_sc_fac, f->d_row_off,
                                                     f->d_row_idx, f->at.pos, f->at.charge, rep_of, f->d_reps,
                                                     f->d_rows, f->at.force, f->d_esc);
  f->launches++;
}

void launch_water(rbmd_force* f, cudaStream_t s) {
  if (!f->is_cvff()) return;
  if (f->topo) { launch_bonded(f, s); return; }
  if (f->n_mol == 0) return;
  WaterParams wp;
  wp.n_mol = (int)f->n_mol;
  wp.bond_k = f->bond_k;
  wp.bond_r0 = f->bond_r0;
  wp.angle_k = f->angle_k;
  wp.angle_theta0_rad = f->angle_t0 * M_PI / 180.0;
  wp.coul_const = 332.06371;
  k_water_extras<<<(wp.n_mol + 127) / 128, 128, 0, s>>>(wp, f->d_hoh, f->at.pos, f->at.charge,
                                                        f->nrep > 1 ? f->d_rep_of : nullptr, f->d_reps,
                                                        f->at.force, f->d_ebond, f->d_eangle, f->d_ewcoul);
  f->launches++;
}

// Cell sort + list build of a Verlet-skin step captured into a graph: whether any replica
// rebuilds is decided on the device (the drift kernel's skin check), so the two run in the body
// of an IF conditional node that k_open_rebuild opens only on rebuild steps; list-reuse steps
// then skip them instead of launching kernels that read the flag and exit.  The list-reuse
// re-gather stays outside, after the node.  Returns false when nothing was added to the capture
// or only an empty node (the caller then launches the two directly, after it); a failure past
// that point sets cond_failed, and the step is captured again without the node.
template <class R>
bool launch_rebuild_conditional(rbmd_force* f, cudaStream_t s, bool bin) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  if (cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd) != cudaSuccess || cs != cudaStreamCaptureStatusActive)
    return false;
  if (!f->cstream && cudaStreamCreateWithFlags(&f->cstream, cudaStreamNonBlocking) != cudaSuccess) return false;
  cudaGraphConditionalHandle h;
  if (cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault) != cudaSuccess) return false;
  k_open_rebuild<<<1, 1, 0, s>>>(h, f->d_rebuild + f->nrep);
  f->launches++;
  if (cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd) != cudaSuccess) {
    f->cond_failed = true;
    return true;
  }
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeIf;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  if (cudaGraphAddNode(&node, g, deps, nd, &cp) != cudaSuccess) {
    f->cond_failed = true;
    return true;
  }
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  if (cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies) != cudaSuccess) {
    f->cond_failed = true;
    return true;
  }
  if (cudaStreamBeginCaptureToGraph(f->cstream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) !=
      cudaSuccess)
    return false;   // an empty body: the sort and list follow the node unconditionally
  launch_sort<R>(f, f->cstream, bin, false);
  launch_nlist<R>(f, f->cstream);
  cudaGraph_t out = nullptr;
  if (cudaStreamEndCapture(f->cstream, &out) != cudaSuccess) f->cond_failed = true;
  return true;
}

// Force evaluation from the current master positions: the k-space chain forks onto the side
// stream, the cell sort / neighbour list / near pass / intramolecular terms run on the caller's
// stream, and the far force is folded in after the join.
template <class R>
void launch_force_tail(rbmd_force* f, cudaStream_t s, bool bin, bool regather) {
  const bool kspace = f->is_rbe();
  if (kspace) {
    cudaEventRecord(f->ev_fork, s);
    launch_kspace<R>(f, f->side, f->ev_fork);
  }
  // a captured Verlet-skin step: sort + list in a conditional node (not for RBL, whose list is
  // rebuilt every step)
  const bool cond = f->capturing && f->cond_rebuild && f->skin > 0 && !f->is_rbl() && bin &&
                    launch_rebuild_conditional<R>(f, s, bin);
  if (cond) {
    if (regather) launch_regather<R>(f, s);
  } else {
    launch_sort<R>(f, s, bin, regather);
  }
  if (f->is_rbl()) {
    launch_rbl_list<R>(f, s);
    PhaseScope ps(f, kPhForce, s);
    launch_rbl_force<R>(f, s);
  } else {
    if (!cond) launch_nlist<R>(f, s);
    PhaseScope ps(f, kPhForce, s);
    if (f->is_eam()) launch_eam<R>(f, s);
    else launch_near<R>(f, s);
  }
  {
    PhaseScope ps(f, kPhMol, s);
    launch_water(f, s);
  }
  if (kspace) {
    cudaStreamWaitEvent(s, f->ev_join, 0);
    if (f->nq > 0) {
      k_add_far<<<(3 * f->nq + 255) / 256, 256, 0, s>>>(f->nq, f->d_qidx, f->d_far, f->at.force, f->d_status);
      f->launches++;
    }
  }
  if (f->tstat == 4 && f->at.vel) {   // Langevin force on top of the total force
    LangevinParams lp;
    lp.n = f->n;
    lp.shared = f->langevin_shared ? 1 : 0;
    lp.gamma = f->langevin_gamma;
    lp.dt = f->dt;
    lp.kBT = f->langevin_shared ? 1.0 : f->u.kB * f->T0;
    lp.fmt2v = f->u.fmt2v;
    lp.mvv2e = f->u.mvv2e;
    for (int d = 0; d < 3; ++d) lp.xi[d] = f->langevin_xi[d];
    lp.seed = f->seed ^ 0x4c616e676576696eull;
    k_langevin<<<(f->n + 255) / 256, 256, 0, s>>>(lp, f->at.vel, f->at.mass, f->d_lstep, f->at.force);
    k_step_inc<<<1, 1, 0, s>>>(f->d_lstep);
    f->launches += 2;
  }
}

template <class R>
void launch_compute(rbmd_force* f, cudaStream_t s) {
  f->want_energy = true;
  f->presampled = false;   // a force call draws the k-set of the current step counter itself
  cudaMemsetAsync(f->d_maxcount, 0, 2 * sizeof(int), s);
  if (f->skin > 0 && f->list_valid) {
    // reuse the list when no atom moved more than skin/2 since it was built
    cudaMemsetAsync(f->d_rebuild, 0, sizeof(int) * (f->nrep + 1), s);
    k_skin_check<<<(f->n + 255) / 256, 256, 0, s>>>(f->n, f->at.pos, f->d_xref,
                                                    f->nrep > 1 ? f->d_rep_of : nullptr, f->d_reps,
                                                    0.25 * f->skin * f->skin, f->d_rebuild, f->nrep);
    f->launches++;
  } else if (f->d_rebuild) {
    cudaMemsetAsync(f->d_rebuild, 1, sizeof(int) * (f->nrep + 1), s);   // nonzero: rebuild
  }
  launch_force_tail<R>(f, s, true, true);
  f->list_valid = true;
}

void launch_compute_any(rbmd_force* f, cudaStream_t s) {
  if (f->fp64) launch_compute<double>(f, s);
  else launch_compute<float>(f, s);
}

// The captured steps bake in buffers, kernel variants and host-side choices (injected
// k-samples, importance weights, proposal, topology); whatever changes one of them drops them,
// and the next multi-step call captures again.
void drop_graphs(rbmd_force* f) {
  f->presampled = false;
  if (f->graph_exec || f->graph_multi) cudaDeviceSynchronize();   // none still in flight
  if (f->graph_exec) cudaGraphExecDestroy(f->graph_exec);
  f->graph_exec = nullptr;
  if (f->graph_multi) cudaGraphExecDestroy(f->graph_multi);
  f->graph_multi = nullptr;
}

rbmd_status grow_list(rbmd_force* f, const int* need) {
  drop_graphs(f);   // buffers move: the captured steps are stale
  auto grown = [](int cur, int want) { return std::max(cur, ((int)(want * 1.2) + 8 + 7) & ~7); };
  if (f->is_rbl()) {
    f->core_cap = grown(f->core_cap, need[0]);
    f->shell_cap = grown(f->shell_cap, need[1]);
    f->cap = f->core_cap + f->shell_cap;
  } else {
    f->cap = ((int)(need[0] * 1.2) + 8 + 7) & ~7;
  }
  dfree(f->d_nbr);
  CK(dalloc(&f->d_nbr, (size_t)f->cap * f->stride));
  return RBMD_OK;
}

// Check the list-capacity flag after a launch sequence; returns 1 when the work must be redone.
rbmd_status check_overflow(rbmd_force* f, cudaStream_t s, bool* redo) {
  *redo = false;
  CK(cudaMemcpyAsync(f->h_status, f->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(f->h_maxcount, f->d_maxcount, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  prof_collect(f);
  if (*f->h_status & kFlagListOverflow) {
    f->list_valid = false;
    rbmd_status st = grow_list(f, f->h_maxcount);
    if (st) return st;
    uint32_t clr = *f->h_status & ~kFlagListOverflow;
    CK(cudaMemcpyAsync(f->d_status, &clr, sizeof clr, cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));
    *redo = true;
  }
  return RBMD_OK;
}

template <class R>
void launch_step(rbmd_force* f, cudaStream_t s) {
  if (f->capturing) cudaEventRecord(f->ev_begin, s);
  const int n = f->n;
  const bool shake = f->shake == "true" && f->n_mol > 0;
  MdParams mp;
  mp.n = n;
  mp.dt = f->dt;
  mp.fmt2v = f->u.fmt2v;
  mp.wrap_flags = (f->shake == "null" || f->init_way == "inbuild") ? 1 : 0;
  mp.save_old = shake ? 1 : 0;
  mp.apply_scale = f->pending_scale ? 1 : 0;
  mp.nh = f->tstat == 3;
  f->want_energy = f->energy_every > 0 && ((f->step_count + 1) % f->energy_every == 0);
  cudaMemsetAsync(f->d_maxcount, 0, 2 * sizeof(int), s);
  const bool skin = f->skin > 0;
  // without a skin the drift bins every step; with one it writes the slot caches (unless SHAKE
  // moves the atoms afterwards) and k_bin bins on rebuild steps only
  if (!skin) cudaMemsetAsync(f->d_cell_count, 0, sizeof(int) * f->ncell_total, s);
  // with a skin the drift kernel decides; a missing or overflowed list forces a rebuild
  if (skin) cudaMemsetAsync(f->d_rebuild, f->list_valid ? 0 : 1, sizeof(int) * (f->nrep + 1), s);
  // (the slot map exists once a cell sort has run: list_valid)
  const bool drift_cache = skin && !shake && f->list_valid;
  // stages 1-2: kick, drift + wrap, bin (binning sees the unconstrained positions, as the
  // reference's locator.SetPosition runs before ConstraintA)
  {
    PhaseScope ps(f, kPhInt, s);
    k_kick_drift<R><<<(n + 255) / 256, 256, 0, s>>>(mp, f->at.pos, f->at.vel, f->at.force, f->at.mass,
                                                    f->at.image, f->nrep > 1 ? f->d_rep_of : nullptr,
                                                    f->d_reps, f->d_lambda, f->d_xold, f->d_vold,
                                                    skin ? nullptr : f->d_cell_of, skin ? nullptr : f->d_cell_count,
                                                    f->d_status, skin ? f->d_xref : nullptr,
                                                    0.25 * f->skin * f->skin, f->d_rebuild, f->nrep,
                                                    f->d_atom_slot,
                                                    f->at.charge,
                                                    drift_cache ? (typename Traits<R>::V4*)f->d_pos4 : nullptr);
    f->launches++;
  }
  if (shake) {
    PhaseScope ps(f, kPhMol, s);
    ShakeParams sp;
    sp.n_mol = (int)f->n_mol;
    sp.dt = f->dt;
    sp.fmt2v = f->u.fmt2v;
    sp.tol = f->shake_tol;
    sp.max_iter = f->shake_max_iter;
    k_shake<<<(sp.n_mol + 127) / 128, 128, 0, s>>>(sp, f->d_hoh, f->at.pos, f->at.vel, f->d_xold,
                                                  f->d_vold, f->at.force, f->at.mass, f->at.image,
                                                  f->nrep > 1 ? f->d_rep_of : nullptr, f->d_reps,
                                                  f->d_status);
    f->launches++;
  }
  // stage 3: force (cell sort of the pre-constraint binning, then list and forces)
  launch_force_tail<R>(f, s, skin, skin && !drift_cache);
  f->list_valid = true;
  // stage 3: kick (+ RATTLE), temperature, thermostat
  PhaseScope ps_int(f, kPhInt, s);
  if (shake) {
    k_kick_ke<<<f->nchunks, 256, 0, s>>>(mp, f->d_chunks, f->at.vel, f->at.force, f->at.mass, 1,
                                        nullptr, nullptr);
    k_rattle<<<((int)f->n_mol + 127) / 128, 128, 0, s>>>((int)f->n_mol, f->d_hoh, f->at.pos, f->at.vel,
                                                         f->at.mass, f->nrep > 1 ? f->d_rep_of : nullptr,
                                                         f->d_reps, f->d_status);
    k_kick_ke<<<f->nchunks, 256, 0, s>>>(mp, f->d_chunks, f->at.vel, f->at.force, f->at.mass, 0,
                                        nullptr, f->d_ke_partial);
    f->launches += 3;
  } else {
    k_kick_ke<<<f->nchunks, 256, 0, s>>>(mp, f->d_chunks, f->at.vel, f->at.force, f->at.mass, 1,
                                        nullptr, f->d_ke_partial);
    f->launches++;
  }
  if (f->tstat == 3) {
    k_kick_ke<<<f->nchunks, 256, 0, s>>>(mp, f->d_chunks, f->at.vel, f->at.force, f->at.mass, 2,
                                        f->d_xi, nullptr);
    f->launches++;
  }
  ThermoParams tp;
  tp.nrep = f->nrep;
  tp.tstat = f->tstat;
  tp.mvv2e = f->u.mvv2e;
  tp.kB = f->u.kB;
  tp.dt = f->dt;
  tp.Tdamp = f->Tdamp;
  tp.T0 = f->T0;
  tp.dof_mode = f->dof_mode;
  k_thermo<<<(f->nrep + 3) / 4, 128, 0, s>>>(tp, f->d_chunk_rep_begin, f->d_ke_partial, f->d_ke,
                                                f->d_T, f->d_lambda, f->d_xi, f->d_reps);
  f->launches++;
  f->pending_scale = (f->tstat == 1 || f->tstat == 2);
  f->step_count++;
}

// n_steps MD steps on stream s.  With execution.cuda_graph (default on) and no per-step host
// decisions (no energy output, no profiling), the first step runs directly (it brings the lazy
// thermostat state and the list flag to their steady values), the next step is captured once on
// an internal stream (the k-space stream joins the capture) and then replayed with one
// cudaGraphLaunch per step on s.  The samplers read the step index from a device counter that
// the k-space chain advances, so every replay draws new k-samples.  The captured step is
// re-captured when the lazy-rescale state differs and dropped when a list grows.
template <class R>
rbmd_status run_steps(rbmd_force* f, int n_steps, cudaStream_t s) {
  const bool graph = f->use_graph && f->energy_every == 0 && !f->prof_on && n_steps > 1;
  if (!graph) {
    for (int k = 0; k < n_steps; ++k) launch_step<R>(f, s);
    if (f->is_rbe()) cudaStreamWaitEvent(s, f->ev_tail, 0);   // the k-space stream's tail joins s
    return RBMD_OK;
  }
  launch_step<R>(f, s);
  if (f->is_rbe()) cudaStreamWaitEvent(s, f->ev_tail, 0);   // graph launches on s follow the whole step
  const int per_step = f->launches;
  if (!f->gstream) CK(cudaStreamCreateWithFlags(&f->gstream, cudaStreamNonBlocking));
  if (!f->ev_begin) CK(cudaEventCreateWithFlags(&f->ev_begin, cudaEventDisableTiming));
  // capture `steps` consecutive steps into *exec (host-side state restored afterwards: the
  // kernels take the step index, rebuild flags and noise counters from device memory)
  auto capture = [&](int steps, cudaGraphExec_t* exec, int* launches) -> rbmd_status {
    const long long sc = f->step_count;
    const bool pend = f->pending_scale;
    const int l0 = f->launches;
    // a second attempt runs without the conditional rebuild node when the first could not
    // build it (cond_failed) or its graph does not capture or instantiate here
    for (int attempt = 0;; ++attempt) {
      cudaGraph_t g = nullptr;
      CK(cudaStreamBeginCapture(f->gstream, cudaStreamCaptureModeThreadLocal));
      f->capturing = true;
      for (int k = 0; k < steps; ++k) launch_step<R>(f, f->gstream);
      if (f->is_rbe()) cudaStreamWaitEvent(f->gstream, f->ev_tail, 0);   // the last step's k-space tail
      f->capturing = false;
      const cudaError_t e = cudaStreamEndCapture(f->gstream, &g);
      *launches = f->launches - l0;
      f->launches = l0;
      f->step_count = sc;
      f->pending_scale = pend;
      cudaError_t ei = e;
      if (e == cudaSuccess && g && !f->cond_failed) ei = cudaGraphInstantiate(exec, g, 0);
      if (g) cudaGraphDestroy(g);
      if (ei == cudaSuccess && g && !f->cond_failed) return RBMD_OK;
      const bool retry = attempt == 0 && f->cond_rebuild;
      f->cond_failed = false;
      f->cond_rebuild = false;
      cudaGetLastError();
      *exec = nullptr;
      if (!retry) {
        std::snprintf(g_last_error, sizeof g_last_error, "step graph: %s",
                      cudaGetErrorString(ei != cudaSuccess ? ei : cudaErrorUnknown));
        return RBMD_ERR_CUDA;
      }
    }
  };
  if (!f->graph_exec || f->graph_pending != f->pending_scale) {
    if (f->graph_exec) cudaGraphExecDestroy(f->graph_exec);
    f->graph_exec = nullptr;
    rbmd_status st = capture(1, &f->graph_exec, &f->graph_launches);
    if (st) return st;
    f->graph_pending = f->pending_scale;
  }
  int remaining = n_steps - 1;
  const int m = f->graph_steps;
  if (m > 1 && remaining >= m) {
    // several steps per graph launch: small systems pay the graph launch once per m steps
    if (!f->graph_multi || f->graph_multi_pending != f->pending_scale) {
      if (f->graph_multi) cudaGraphExecDestroy(f->graph_multi);
      f->graph_multi = nullptr;
      rbmd_status st = capture(m, &f->graph_multi, &f->graph_multi_launches);
      if (st) return st;
      f->graph_multi_pending = f->pending_scale;
    }
    for (; remaining >= m; remaining -= m) {
      CK(cudaGraphLaunch(f->graph_multi, s));
      f->step_count += m;
      f->launches += f->graph_multi_launches;
    }
  }
  for (; remaining > 0; --remaining) {
    CK(cudaGraphLaunch(f->graph_exec, s));
    f->step_count++;
    f->launches += f->graph_launches ? f->graph_launches : per_step;
  }
  return RBMD_OK;
}

rbmd_status parse_config(rbmd_force* f, const char* text) {
  rbmdjson::Value root;
  std::string err;
  if (!text || !rbmdjson::parse(text, root, err)) {
    std::snprintf(g_last_error, sizeof g_last_error, "config: %s", err.c_str());
    return RBMD_ERR_CONFIG;
  }
  using namespace rbmdjson;
  f->ff = rbmdjson::text(root, "hyper_parameters.force_field.type", "LJ/CUT");
  f->potential_file = rbmdjson::text(root, "hyper_parameters.force_field.potential_file", "");
  f->potential_format = rbmdjson::text(root, "hyper_parameters.force_field.potential_format", "");
  f->nbr_type = rbmdjson::text(root, "hyper_parameters.neighbor.type", "VERLETLIST");
  if (f->nbr_type == "VERLET-LIST") f->nbr_type = "VERLETLIST";
  // "ORIGINAL" walks the cells on the fly and leaves the cutoff to the force function
  // (ExecPointLocator::ExecuteOnNeighbor): here a list built with the force function's
  // predicate d^2 < rc^2 instead of the list's rc^2 - d^2 > 1e-4, otherwise a Verlet list
  if (f->nbr_type == "ORIGINAL") {
    f->orig_pred = true;
    f->nbr_type = "VERLETLIST";
  }
  bool found = false;
  f->rc = num(root, "hyper_parameters.neighbor.cut_off", 0.0, &found);
  if (!found || f->rc <= 0) {
    std::snprintf(g_last_error, sizeof g_last_error, "config: neighbor.cut_off missing");
    return RBMD_ERR_CONFIG;
  }
  f->rs = f->nbr_type == "RBL" ? num(root, "hyper_parameters.neighbor.r_core", f->rc) : f->rc;
  f->skin = num(root, "hyper_parameters.neighbor.skin", 0.0);
  f->cap_override = (int)num(root, "hyper_parameters.neighbor.capacity", 0.0);
  {
    const Value* at = root.path("autotune");
    if (at && at->kind == Value::Bool) f->autotune = at->b;
    const int tl = (int)num(root, "tuning.list_block", 0.0), tn = (int)num(root, "tuning.force_block", 0.0);
    auto ok = [](int t) { return t == 64 || t == 128 || t == 256; };
    const Value* tlv = root.path("tuning.list_block");
    if (ok(tl) || (tlv && (tl == 0 || tl == 1))) { f->tpa_list = tl; f->autotune = false; }
    if (ok(tn)) { f->tpa_near = tn; f->autotune = false; }
    const Value* nv = root.path("tuning.near_variant");
    if (nv) f->near_variant = (int)num(root, "tuning.near_variant", 1.0) == 0 ? 0 : 1;
    const int ln = (int)num(root, "tuning.force_lanes", 0.0);
    if (ln == 1 || ln == 4 || ln == 8 || ln == 16 || ln == 32) { f->near_lanes = ln; f->autotune = false; }
    const std::string rl = rbmdjson::text(root, "tuning.rbl_list", "auto");
    if (rl != "warp" && rl != "thread" && rl != "auto") {
      std::snprintf(g_last_error, sizeof g_last_error,
                    "config: tuning.rbl_list must be \"auto\", \"warp\" or \"thread\"");
      return RBMD_ERR_CONFIG;
    }
    f->rbl_list_warp = rl == "warp" ? 1 : (rl == "thread" ? 0 : -1);
    const int rg = (int)num(root, "tuning.rbl_lanes", 0.0);
    if (rg == 1 || rg == 4 || rg == 8 || rg == 16 || rg == 32) f->rbl_lanes = rg;
  }
  f->far = root.path("hyper_parameters.coulomb") != nullptr;
  if (f->far) {
    f->coul_type = rbmdjson::text(root, "hyper_parameters.coulomb.type", "RBE");
    f->P = (int)num(root, "hyper_parameters.coulomb.coulomb_sample_num", 100);
    f->alpha = num(root, "hyper_parameters.coulomb.alpha", 0.1);
    f->kmax = (int)num(root, "hyper_parameters.coulomb.kmax", 2);
    f->seed = (unsigned long long)num(root, "hyper_parameters.coulomb.seed", 20240101.0);
    f->proposal = rbmdjson::text(root, "hyper_parameters.coulomb.proposal", "gauss");
    if (f->proposal != "gauss" && f->proposal != "gauss_iid" && f->proposal != "learned") {
      std::snprintf(g_last_error, sizeof g_last_error, "config: unknown coulomb.proposal %s", f->proposal.c_str());
      return RBMD_ERR_CONFIG;
    }
  }
  f->shake = rbmdjson::text(root, "hyper_parameters.extend.fix_shake", "null");
  f->shake_tol = num(root, "hyper_parameters.extend.shake_tolerance", 1e-5);
  f->shake_max_iter = (int)num(root, "hyper_parameters.extend.shake_max_iter", 5000);
  {
    // MDApplication.cpp:157-163: a non-empty special_bonds list turns on the special-bond path
    // (the reference parses it as integers, Extend.cpp:39; fractional weights are kept here)
    std::vector<double> sb = nums(root, "hyper_parameters.extend.special_bonds");
    f->special = !sb.empty();
    for (int k = 0; k < 3; ++k) f->special_w[k] = k < (int)sb.size() ? sb[k] : 0.0;
  }
  std::string prec = rbmdjson::text(root, "precision", "fp32");
  f->fp64 = prec == "fp64" || prec == "FP64" || prec == "double";
  if (root.path("init_configuration.inbuild")) {
    f->init_way = "inbuild";
    f->unit = rbmdjson::text(root, "init_configuration.inbuild.unit", "LJ");
  } else {
    f->init_way = "read_data";
    f->unit = rbmdjson::text(root, "init_configuration.read_data.unit", "LJ");
  }
  f->u = units_for(f->unit);
  f->dt = num(root, "execution.timestep", 0.005);
  f->energy_every = (int)num(root, "outputs.thermo_out.interval", 0.0);
  {
    const Value* kp = root.path("execution.kspace_priority");
    if (kp && kp->kind == Value::Bool) f->kspace_priority = kp->b;
    const Value* g = root.path("execution.cuda_graph");
    if (g && g->kind == Value::Bool) f->use_graph = g->b;
    const int gs = (int)num(root, "execution.graph_steps", 8.0);
    if (gs < 1 || gs > 64) {
      std::snprintf(g_last_error, sizeof g_last_error, "config: execution.graph_steps must be 1..64");
      return RBMD_ERR_CONFIG;
    }
    f->graph_steps = gs;
  }
  std::vector<double> T = nums(root, "execution.temperature");
  f->T0 = T.size() > 0 ? T[0] : 1.0;
  f->Tdamp = T.size() > 2 ? T[2] : 1.0;
  std::string ens = rbmdjson::text(root, "execution.ensemble", "NVT");
  f->tctrl = rbmdjson::text(root, "execution.temp_ctrl_type", "");
  f->tstat = 0;
  if (ens != "NVE") {
    if (f->tctrl == "BERENDSEN") f->tstat = 1;
    else if (f->tctrl == "TEMP_RESCALE") f->tstat = 2;
    else if (f->tctrl == "NOSE_HOOVER") f->tstat = 3;
    else if (f->tctrl == "LANGEVIN") f->tstat = 4;
  }
  f->langevin_gamma = num(root, "execution.langevin_gamma", 100.0);
  {
    const Value* lr = root.path("compat.langevin_reference");
    f->langevin_shared = lr && lr->kind == Value::Bool && lr->b;
    // the reference draws its single noise vector once per run (ExecutionNVT.cpp:346-352)
    std::mt19937_64 rng(f->seed * 0x9E3779B97F4A7C15ull + 29);
    std::normal_distribution<double> nd(0.0, 1.0);
    for (int d = 0; d < 3; ++d) f->langevin_xi[d] = nd(rng);
  }
  if (f->init_way == "inbuild") f->dof_mode = 3;
  else if (f->shake == "true") f->dof_mode = 1;
  else if (f->shake == "false") f->dof_mode = 2;
  else f->dof_mode = 0;
  // The Verlet-list near Coulomb of the reference omits qqr2e (RunWorklet.cpp:218,233) while its
  // RBL path applies it (:807).  Default: physical force (x qqr2e); compat flag restores the
  // reference's Verlet behaviour.
  bool compat_noq = false;
  const Value* c = root.path("compat.verlet_coul_no_qqr2e");
  if (c && c->kind == Value::Bool) compat_noq = c->b;
  f->near_coul_scale = compat_noq ? 1.0 : f->u.qqr2e;
  if (f->ff != "LJ/CUT" && f->ff != "LJ/CUT/COUL/LONG" && f->ff != "CVFF" && f->ff != "EAM") {
    std::snprintf(g_last_error, sizeof g_last_error, "config: unknown force_field.type %s", f->ff.c_str());
    return RBMD_ERR_CONFIG;
  }
  if (f->ff == "LJ/CUT" || f->ff == "EAM") f->far = false;
  if (f->far && f->coul_type != "RBE" && f->coul_type != "EWALD") {
    std::snprintf(g_last_error, sizeof g_last_error, "config: unknown coulomb.type %s", f->coul_type.c_str());
    return RBMD_ERR_CONFIG;
  }
  if (f->nbr_type != "VERLETLIST" && f->nbr_type != "RBL") {
    std::snprintf(g_last_error, sizeof g_last_error,
                  "config: neighbor.type %s is not provided by this build (VERLETLIST, ORIGINAL, RBL)",
                  f->nbr_type.c_str());
    return RBMD_ERR_CONFIG;
  }
  // RBL (Neighbor.cpp:40-44): r_core and neighbor_sample_num; the shell subsample follows the
  // traversal of the current positions, so the lists are rebuilt at every force evaluation
  if (f->nbr_type == "RBL") {
    f->rbl_sample_num = num(root, "hyper_parameters.neighbor.neighbor_sample_num", 100.0);
    if (!(f->rs > 0) || !(f->rs < f->rc) || !(f->rbl_sample_num >= 1)) {
      std::snprintf(g_last_error, sizeof g_last_error,
                    "config: RBL needs 0 < r_core < cut_off and neighbor_sample_num >= 1");
      return RBMD_ERR_CONFIG;
    }
    if (f->skin > 0) {
      std::snprintf(g_last_error, sizeof g_last_error, "config: neighbor.skin applies to VERLETLIST only");
      return RBMD_ERR_CONFIG;
    }
  }
  // reference quirks kept behind switches (the defaults are the physical forces):
  //  * compat.rbl_erf_table: RBL Coulomb G from the reference's ERF table, built for alpha 0.1 and
  //    holding one value per distance bucket (ExecStaticTable.h:96-135, RunWorklet.cpp:772-773);
  //  * compat.rbl_drop_shell_coulomb: the shell Coulomb term is computed and discarded
  //    (RunWorklet.cpp:782);
  //  * compat.eam_verlet_pair_vector: the Verlet EAM force on MinDistanceVec(p_j, p_i)
  //    (RunWorklet.cpp:402), which reverses it (the RBL pass uses p_i - p_j, :1180, and so do the
  //    ORIGINAL type's on-the-fly worklets, :419-524, which the flag therefore leaves alone);
  //  * compat.special_bonds_integer: extend.special_bonds read as integers, as Extend does
  //    (GetVectorValueJudge<int>, rbmd/framework/hyperparameters/Extend.cpp:39): 0.5 becomes 0.
  auto flag = [&](const char* key) {
    const Value* v = root.path(key);
    return v && v->kind == Value::Bool && v->b;
  };
  f->rbl_table = flag("compat.rbl_erf_table");
  f->rbl_shell_coul = !flag("compat.rbl_drop_shell_coulomb");
  f->eam_ref_sign = flag("compat.eam_verlet_pair_vector") && !f->orig_pred;
  if (flag("compat.special_bonds_integer"))
    for (double& w : f->special_w) w = std::trunc(w);
  if (f->P < 1 || f->P > 65536) return RBMD_ERR_CONFIG;
  return RBMD_OK;
}

// Per-type LJ tables in the reference's float arithmetic: -24*sqrt(eps_i*eps_j) and
// ((sigma_i + sigma_j)/2)^6 as ComputeLJForce forms them (ExecForceFunction.h:74-96).
void fill_lj(rbmd_force* f, int nt, const double* eps, const double* sig) {
  f->ntypes = nt;
  bool same = true;
  for (int a = 1; a < nt; ++a) same = same && eps[a] == eps[0] && sig[a] == sig[0];
  f->nt_eff = same ? 1 : nt;
  for (int a = 0; a < nt; ++a)
    for (int b = 0; b < nt; ++b) {
      const float ea = (float)eps[a], eb = (float)eps[b], sa = (float)sig[a], sb = (float)sig[b];
      const float sij = (sa + sb) / 2;
      f->ljt_h.lj24_f[a * nt + b] = (float)(-24) * std::sqrt(ea * eb);
      f->ljt_h.sig6_f[a * nt + b] = sij * sij * sij * sij * sij * sij;
      const double sd = (sig[a] + sig[b]) / 2;
      f->ljt_h.lj24_d[a * nt + b] = -24.0 * std::sqrt(eps[a] * eps[b]);
      f->ljt_h.sig6_d[a * nt + b] = sd * sd * sd * sd * sd * sd;
    }
}

rbmd_status upload_ksamples(rbmd_force* f, const int32_t* m_xyz) {
  const int recb = f->fp64 ? sizeof(KRec64) : sizeof(KRec32);
  std::vector<char> buf((size_t)f->Ptot * recb, 0);
  for (int g = 0; g < f->Ptot; ++g) {
    int* rec = reinterpret_cast<int*>(buf.data() + (size_t)g * recb);
    rec[0] = m_xyz[3 * g];
    rec[1] = m_xyz[3 * g + 1];
    rec[2] = m_xyz[3 * g + 2];
    if (rec[0] == 0 && rec[1] == 0 && rec[2] == 0) return RBMD_ERR_ARG;
  }
  std::vector<int> krep(f->Ptot);
  for (int g = 0; g < f->Ptot; ++g) krep[g] = g / f->P;
  CK(cudaMemcpy(f->d_krep, krep.data(), sizeof(int) * f->Ptot, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(f->d_krec, buf.data(), buf.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(f->d_kvec, m_xyz, sizeof(int) * 3 * f->Ptot, cudaMemcpyHostToDevice));
  f->injected = true;
  return RBMD_OK;
}

// Own autotuner: times every threads-per-block choice of the list build and of the force pass
// (three timed launches each after a warm-up, best taken) on the bound system and keeps the
// fastest.
template <class R>
rbmd_status autotune_impl(rbmd_force* f, cudaStream_t s) {
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  const bool prof = f->prof_on;
  f->prof_on = false;
  const int cand[3] = {64, 128, 256};
  // rebuild pattern of the timed list builds: every replica of a single system; in a batch with
  // a Verlet skin about one replica in five rebuilds per step (each decides alone), and the list
  // variants rank differently on such partial rebuilds than on full ones, so one in five is
  // flagged there
  std::vector<int> rb_pattern(f->nrep + 1, 1);
  if (f->nrep > 1 && f->skin > 0)
    for (int r = 0; r < f->nrep; ++r) rb_pattern[r] = r % 5 == 0 ? 1 : 0;
  auto best_of = [&](auto launch) -> float {
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
      if (f->d_rebuild)
        cudaMemcpyAsync(f->d_rebuild, rb_pattern.data(), sizeof(int) * (f->nrep + 1), cudaMemcpyHostToDevice, s);
      cudaEventRecord(a, s);
      launch();
      cudaEventRecord(b, s);
      cudaEventSynchronize(b);
      float ms = 0;
      cudaEventElapsedTime(&ms, a, b);
      if (rep > 0) best = std::min(best, ms);
    }
    return best;
  };
  float bl = 1e30f, bn = 1e30f;
  int tl = f->tpa_list, tn = f->tpa_near;
  const int lcand[5] = {0, 1, 64, 128, 256};   // 0: the staged build, 1: warp per atom
  for (int t : lcand) {
    if (t == 0 && f->nsegs == 0) continue;
    if (t == 1 && f->num_cycles != 1) continue;
    f->tpa_list = t;
    const float ms = best_of([&] { launch_nlist<R>(f, s); });
    if (ms < bl) { bl = ms; tl = t; }
  }
  f->tpa_list = tl;
  int tg = f->near_lanes;
  const int gcand[5] = {1, 4, 8, 16, 32};
  for (int g : gcand) {
    if (g > 1 && f->is_eam()) continue;
    for (int t : cand) {
      if (g > 1 && t != 256) continue;   // grouped variants run 256-thread blocks
      f->tpa_near = t;
      f->near_lanes = g;
      const float ms = best_of([&] {
        if (f->is_eam()) launch_eam<R>(f, s);
        else launch_near<R>(f, s);
      });
      if (ms < bn) { bn = ms; tn = t; tg = g; }
    }
  }
  f->near_lanes = tg;
  f->tpa_near = tn;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  f->prof_on = prof;
  CK(cudaGetLastError());
  f->tuned = true;
  return RBMD_OK;
}

}  // namespace

// ==========================================================================================
// C ABI
// ==========================================================================================
extern "C" {

const char* rbmd_version(void) { return "rbmd-b200 0.1 (sm_100a)"; }

const char* rbmd_last_error(void) { return g_last_error; }

rbmd_status rbmd_force_create(const char* json_text, int32_t n_replicas, const rbmd_box* boxes,
                              rbmd_force** out) {
  if (!out || !boxes || n_replicas < 1) return RBMD_ERR_ARG;
  *out = nullptr;
  rbmd_force* f = new rbmd_force();
  rbmd_status st = parse_config(f, json_text);
  if (st) { delete f; return st; }
  f->nrep = n_replicas;
  f->boxes.assign(boxes, boxes + n_replicas);
  for (int r = 0; r < n_replicas; ++r)
    for (int d = 0; d < 3; ++d)
      if (!(boxes[r].hi[d] > boxes[r].lo[d])) { delete f; return RBMD_ERR_ARG; }
  const double one = 1.0;
  fill_lj(f, 1, &one, &one);
  if (f->is_eam() && !f->potential_file.empty()) {
    if (eam_load(f->potential_file, f->eam_h, f->potential_format) != 0) {
      std::snprintf(g_last_error, sizeof g_last_error, "cannot read EAM potential file %s",
                    f->potential_file.c_str());
      delete f;
      return RBMD_ERR_FILE;
    }
    f->eam_loaded = true;
  }
  *out = f;
  return RBMD_OK;
}

rbmd_status rbmd_force_set_pair_coeffs(rbmd_force* f, int32_t n_types, const double* epsilon,
                                       const double* sigma) {
  if (f) drop_graphs(f);
  if (!f || !epsilon || !sigma || n_types < 1 || n_types > kMaxReplicaTypes) return RBMD_ERR_ARG;
  fill_lj(f, n_types, epsilon, sigma);
  f->have_pair_coeffs = true;
  if (f->d_ljt) CK(cudaMemcpy(f->d_ljt, &f->ljt_h, sizeof(LJTable), cudaMemcpyHostToDevice));
  return RBMD_OK;
}

rbmd_status rbmd_force_load_funcfl(rbmd_force* f, const char* path) {
  if (f) drop_graphs(f);
  if (!f || !path) return RBMD_ERR_ARG;
  if (eam_load(path, f->eam_h, f->potential_format) != 0) return RBMD_ERR_FILE;
  f->eam_loaded = true;
  f->potential_file = path;
  return RBMD_OK;
}

rbmd_status rbmd_force_set_water(rbmd_force* f, int64_t n_mol, const int32_t* hoh, double bond_k,
                                 double bond_r0, double angle_k, double angle_theta0_deg) {
  if (f) drop_graphs(f);
  if (!f || n_mol < 0 || (n_mol > 0 && !hoh)) return RBMD_ERR_ARG;
  f->n_mol = n_mol;
  f->hoh_h.assign(hoh, hoh + 3 * n_mol);
  f->bond_k = bond_k;
  f->bond_r0 = bond_r0;
  f->angle_k = angle_k;
  f->angle_t0 = angle_theta0_deg;
  if (f->bound) {
    dfree(f->d_hoh);
    CK(dalloc(&f->d_hoh, (size_t)3 * n_mol));
    CK(cudaMemcpy(f->d_hoh, f->hoh_h.data(), sizeof(int) * 3 * n_mol, cudaMemcpyHostToDevice));
    dfree(f->d_ebond); dfree(f->d_eangle); dfree(f->d_ewcoul);
    CK(dalloc(&f->d_ebond, (size_t)n_mol));
    CK(dalloc(&f->d_eangle, (size_t)n_mol));
    CK(dalloc(&f->d_ewcoul, (size_t)n_mol));
  }
  return RBMD_OK;
}

// Device copies of the topology tables (at bind, or at set_topology once bound).
static rbmd_status upload_topology(rbmd_force* f) {
  free_topology(f);
  if (!f->topo) return RBMD_OK;
  if (f->topo_n != f->n) {
    std::snprintf(g_last_error, sizeof g_last_error, "topology has %lld atoms, bound arrays %d",
                  (long long)f->topo_n, f->n);
    return RBMD_ERR_ARG;
  }
  auto upi = [&](const std::vector<int32_t>& v, int** d) -> cudaError_t {
    cudaError_t e = dalloc(d, v.size());
    if (e == cudaSuccess && !v.empty())
      e = cudaMemcpy(*d, v.data(), sizeof(int) * v.size(), cudaMemcpyHostToDevice);
    return e;
  };
  auto upd = [&](const std::vector<double>& v, double** d) -> cudaError_t {
    cudaError_t e = dalloc(d, v.size());
    if (e == cudaSuccess && !v.empty())
      e = cudaMemcpy(*d, v.data(), sizeof(double) * v.size(), cudaMemcpyHostToDevice);
    return e;
  };
  CK(upi(f->term_atom_h, &f->d_term_atom));
  CK(upi(f->tmult_h, &f->d_tmult));
  CK(upd(f->tk_h, &f->d_tk));
  CK(upd(f->ta_h, &f->d_ta));
  CK(upi(f->sc_off_h, &f->d_sc_off));
  CK(upi(f->sc_id_h, &f->d_sc_id));
  CK(upd(f->sc_fac_h, &f->d_sc_fac));
  CK(upi(f->row_off_h, &f->d_row_off));
  CK(upi(f->row_idx_h, &f->d_row_idx));
  CK(dalloc(&f->d_rows, 3 * f->term_atom_h.size()));
  CK(dalloc(&f->d_eterm, (size_t)(f->topo_nb + f->topo_na + f->topo_nd)));
  CK(dalloc(&f->d_esc, (size_t)f->n));
  CK(cudaMemset(f->d_esc, 0, sizeof(double) * f->n));
  CK(cudaMemset(f->d_eterm, 0, sizeof(double) * std::max(1, f->topo_nb + f->topo_na + f->topo_nd)));
  if (f->special) {
    CK(upi(f->sp_off_h, &f->d_sp_off));
    CK(upi(f->sp_id_h, &f->d_sp_id));
    CK(upd(f->sp_w_h, &f->d_sp_wd));
    std::vector<float> wf(f->sp_w_h.begin(), f->sp_w_h.end());
    CK(dalloc(&f->d_sp_wf, wf.size()));
    if (!wf.empty()) CK(cudaMemcpy(f->d_sp_wf, wf.data(), sizeof(float) * wf.size(), cudaMemcpyHostToDevice));
    CK(upi(f->comp_h, &f->d_comp));
  }
  return RBMD_OK;
}

rbmd_status rbmd_force_set_topology(rbmd_force* f, const rbmd_topology* t) {
  if (f) drop_graphs(f);
  if (!f || !t || t->n_atoms < 1 || !t->molecule || t->n_bonds < 0 || t->n_angles < 0 || t->n_dihedrals < 0)
    return RBMD_ERR_ARG;
  if (!f->is_cvff()) {   // the reference adds intramolecular terms for "CVFF" only (ExecutionNVT.cpp:199-215)
    std::snprintf(g_last_error, sizeof g_last_error, "topology: force_field.type %s has no bonded terms (CVFF does)",
                  f->ff.c_str());
    return RBMD_ERR_STATE;
  }
  const int64_t n = t->n_atoms;
  const int64_t nb = t->n_bonds, na = t->n_angles, nd = f->special ? t->n_dihedrals : 0;
  if ((nb && (!t->bonds || !t->bond_type || !t->bond_coeffs)) ||
      (na && (!t->angles || !t->angle_type || !t->angle_coeffs)) ||
      (nd && (!t->dihedrals || !t->dihedral_type || !t->dihedral_coeffs)))
    return RBMD_ERR_ARG;
  if (2 * nb + 3 * na + 4 * nd >= (1LL << 31)) return RBMD_ERR_ARG;
  auto bad_ids = [&](const int32_t* a, int64_t cnt) {
    for (int64_t k = 0; k < cnt; ++k)
      if (a[k] < 0 || a[k] >= n) return true;
    return false;
  };
  auto bad_types = [&](const int32_t* a, int64_t cnt, int32_t ntypes) {
    for (int64_t k = 0; k < cnt; ++k)
      if (a[k] < 0 || a[k] >= ntypes) return true;
    return false;
  };
  if (bad_ids(t->bonds, 2 * nb) || bad_ids(t->angles, 3 * na) || (nd && bad_ids(t->dihedrals, 4 * nd)) ||
      bad_types(t->bond_type, nb, t->n_bond_types) || bad_types(t->angle_type, na, t->n_angle_types) ||
      (nd && bad_types(t->dihedral_type, nd, t->n_dihedral_types))) {
    std::snprintf(g_last_error, sizeof g_last_error, "topology: atom id or type out of range");
    return RBMD_ERR_ARG;
  }
  // terms: packed atoms and per-term coefficients
  f->topo_n = n;
  f->topo_nb = (int)nb; f->topo_na = (int)na; f->topo_nd = (int)nd;
  f->term_atom_h.assign(t->bonds, t->bonds + 2 * nb);
  f->term_atom_h.insert(f->term_atom_h.end(), t->angles, t->angles + 3 * na);
  if (nd) f->term_atom_h.insert(f->term_atom_h.end(), t->dihedrals, t->dihedrals + 4 * nd);
  const int64_t nterm = nb + na + nd;
  f->tk_h.assign(nterm, 0.0);
  f->ta_h.assign(nterm, 0.0);
  f->tmult_h.assign(nterm, 0);
  for (int64_t b = 0; b < nb; ++b) {
    f->tk_h[b] = t->bond_coeffs[2 * t->bond_type[b]];
    f->ta_h[b] = t->bond_coeffs[2 * t->bond_type[b] + 1];
  }
  for (int64_t a = 0; a < na; ++a) {
    f->tk_h[nb + a] = t->angle_coeffs[2 * t->angle_type[a]];
    f->ta_h[nb + a] = t->angle_coeffs[2 * t->angle_type[a] + 1] * M_PI / 180.0;
  }
  for (int64_t d = 0; d < nd; ++d) {
    const double* c = t->dihedral_coeffs + 3 * t->dihedral_type[d];
    f->tk_h[nb + na + d] = c[0];
    f->ta_h[nb + na + d] = (int)c[1] == 1 ? 1.0 : -1.0;   // cos_shift (ComputeDihedralHarmonicWorklet)
    f->tmult_h[nb + na + d] = (int)c[2];
  }
  // rows of each atom, ascending (bonds, angles, dihedrals)
  const int64_t nrow = (int64_t)f->term_atom_h.size();
  f->row_off_h.assign(n + 1, 0);
  for (int64_t e = 0; e < nrow; ++e) f->row_off_h[f->term_atom_h[e] + 1]++;
  for (int64_t a = 0; a < n; ++a) f->row_off_h[a + 1] += f->row_off_h[a];
  f->row_idx_h.assign(nrow, 0);
  {
    std::vector<int32_t> cur(f->row_off_h.begin(), f->row_off_h.end() - 1);
    for (int64_t e = 0; e < nrow; ++e) f->row_idx_h[cur[f->term_atom_h[e]]++] = (int32_t)e;
  }
  // molecules (ids may be sparse): members of each, in atom order
  std::unordered_map<int32_t, std::vector<int32_t>> members;
  for (int64_t a = 0; a < n; ++a) members[t->molecule[a]].push_back((int32_t)a);
  // special-bond lists (ModelFileInitCondition::SetSpecialBonds), reduced to one entry per partner
  // carrying the weight of its last occurrence, the one the reference's pair loops keep
  std::vector<std::vector<std::pair<int32_t, double>>> sp(f->special ? n : 0);
  if (f->special) {
    std::vector<std::vector<int32_t>> adj(n);
    for (int64_t b = 0; b < nb; ++b) {
      adj[t->bonds[2 * b]].push_back(t->bonds[2 * b + 1]);
      adj[t->bonds[2 * b + 1]].push_back(t->bonds[2 * b]);
    }
    for (int64_t a = 0; a < n; ++a) {
      std::vector<std::pair<int32_t, double>> raw;
      for (int32_t k1 : adj[a]) {
        raw.push_back({k1, f->special_w[0]});
        for (int32_t k2 : adj[k1]) {
          if (k2 == a) continue;
          raw.push_back({k2, f->special_w[1]});
          for (int32_t k3 : adj[k2]) {
            if (k3 == k1) continue;
            raw.push_back({k3, f->special_w[2]});
          }
        }
      }
      for (size_t k = 0; k < raw.size(); ++k) {
        if (raw[k].first == a) continue;   // never a pair partner
        bool later = false;
        for (size_t l = k + 1; l < raw.size() && !later; ++l) later = raw[l].first == raw[k].first;
        if (!later) sp[a].push_back(raw[k]);
      }
    }
    f->sp_off_h.assign(n + 1, 0);
    f->sp_id_h.clear();
    f->sp_w_h.clear();
    for (int64_t a = 0; a < n; ++a) {
      for (auto& pr : sp[a])
        if (pr.second != 1.0) { f->sp_id_h.push_back(pr.first); f->sp_w_h.push_back(pr.second); }
      f->sp_off_h[a + 1] = (int32_t)f->sp_id_h.size();
    }
    // bond-graph components: special partners always share one, so the near passes look up
    // weights only for pairs inside a component
    std::vector<int32_t> par(n);
    for (int64_t a = 0; a < n; ++a) par[a] = (int32_t)a;
    std::function<int32_t(int32_t)> root = [&](int32_t x) {
      while (par[x] != x) { par[x] = par[par[x]]; x = par[x]; }
      return x;
    };
    for (int64_t b = 0; b < nb; ++b) {
      const int32_t r1 = root(t->bonds[2 * b]), r2 = root(t->bonds[2 * b + 1]);
      if (r1 != r2) par[std::max(r1, r2)] = std::min(r1, r2);
    }
    f->comp_h.assign(n, 0);
    for (int64_t a = 0; a < n; ++a) f->comp_h[a] = root((int32_t)a);
  }
  // intramolecular Coulomb correction lists
  f->sc_off_h.assign(n + 1, 0);
  f->sc_id_h.clear();
  f->sc_fac_h.clear();
  for (int64_t a = 0; a < n; ++a) {
    const auto& g = members.at(t->molecule[a]);
    if (g.size() >= 3) {
      if (!f->special) {
        for (int32_t j : g)
          if (j != a) { f->sc_id_h.push_back(j); f->sc_fac_h.push_back(1.0); }
      } else {
        for (auto& pr : sp[a])
          if (pr.second != 1.0 && t->molecule[pr.first] == t->molecule[a]) {
            f->sc_id_h.push_back(pr.first);
            f->sc_fac_h.push_back(1.0 - pr.second);
          }
      }
    }
    if (f->sc_id_h.size() >= (size_t)1 << 31) {
      std::snprintf(g_last_error, sizeof g_last_error, "topology: intramolecular pair list too long");
      return RBMD_ERR_ARG;
    }
    f->sc_off_h[a + 1] = (int32_t)f->sc_id_h.size();
  }
  f->topo = true;
  if (f->bound) {
    rbmd_status st = upload_topology(f);
    if (st) return st;
    f->list_valid = false;
  }
  return RBMD_OK;
}

rbmd_status rbmd_force_bind(rbmd_force* f, const rbmd_atoms_dev* a) {
  if (!f || !a || a->n_atoms < 1 || !a->pos || !a->force) return RBMD_ERR_ARG;
  if (a->n_atoms >= (1LL << (31 - kShiftBits))) return RBMD_ERR_ARG;
  const int nrep = a->n_replicas < 1 ? 1 : a->n_replicas;
  if (nrep != f->nrep) return RBMD_ERR_ARG;
  if (f->is_eam() && !f->eam_loaded) return RBMD_ERR_STATE;
  free_all(f);
  {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && sms > 0)
      f->num_sms = sms;
  }
  f->at = *a;
  f->n = (int)a->n_atoms;
  f->rep_off.assign(nrep + 1, 0);
  if (nrep == 1) {
    f->rep_off[1] = f->n;
  } else {
    if (!a->replica_offsets) return RBMD_ERR_ARG;
    for (int r = 0; r <= nrep; ++r) f->rep_off[r] = a->replica_offsets[r];
    if (f->rep_off[0] != 0 || f->rep_off[nrep] != f->n) return RBMD_ERR_ARG;
    for (int r = 0; r < nrep; ++r)
      if (f->rep_off[r + 1] <= f->rep_off[r]) return RBMD_ERR_ARG;
  }
  f->at.replica_offsets = nullptr;
  // replica geometry, cells and k ranges
  f->reps_h.assign(nrep, RepDev{});
  int cell_base = 0;
  for (int r = 0; r < nrep; ++r) {
    RepDev& rp = f->reps_h[r];
    int ncyc = 1;
    setup_replica(f->boxes[r], f->list_cut(), f->nbr_type == "RBL" ? f->rs : f->list_cut(), f->fp64, rp,
                  ncyc);
    f->num_cycles = ncyc;
    rp.cell_base = cell_base;
    cell_base += rp.ncell;
    rp.atom_begin = (int)f->rep_off[r];
    rp.atom_end = (int)f->rep_off[r + 1];
    rp.P = f->P;
    rp.k_begin = r * f->P;
    double L[3] = {rp.box_d[0], rp.box_d[1], rp.box_d[2]};
    rp.S = rbe_S(f->alpha, L);
  }
  f->ncell_total = cell_base;
  f->stride = (f->n + 31) & ~31;
  // MinDistanceVec is the identity for listed pairs when every axis has >= 3 cells
  f->minimg = false;
  for (int r = 0; r < nrep; ++r)
    for (int d = 0; d < 3; ++d)
      if (f->reps_h[r].dims[d] < 3) f->minimg = true;
  // list capacity from the densest replica (reference: rho * ceil(4/3 pi rc^3) + 1,
  // ExecutionMD.cpp:683); a margin absorbs fluctuations, overflow triggers regrowth.
  double rho_max = 0;
  for (int r = 0; r < nrep; ++r)
    rho_max = std::max(rho_max, (f->rep_off[r + 1] - f->rep_off[r]) / f->reps_h[r].volume);
  const double lc = f->list_cut();
  f->cap = ((int)(1.5 * rho_max * 4.0 / 3.0 * M_PI * lc * lc * lc) + 32 + 7) & ~7;
  if (f->cap_override > 0) f->cap = f->cap_override;
  if (f->is_rbl()) {
    // pice per replica from the reference's sizing (ExecutionMD.cpp:460-801); capacities from
    // the density with a margin (the reference's rs_num / rc_num rows have no overflow check)
    int pice_min = 1 << 30;
    for (int r = 0; r < nrep; ++r) {
      int64_t z[3];
      rbl_sizes(f, r, z);
      if (z[2] < 1 || z[2] > (1 << 20)) {
        std::snprintf(g_last_error, sizeof g_last_error, "RBL: pice_num %lld out of range", (long long)z[2]);
        return RBMD_ERR_CONFIG;
      }
      f->reps_h[r].rbl_pice = (int)z[2];
      pice_min = std::min(pice_min, (int)z[2]);
      if (r == 0) std::memcpy(f->rbl_sizes_h, z, sizeof z);
    }
    const double rs3 = f->rs * f->rs * f->rs, rc3 = f->rc * f->rc * f->rc;
    f->core_cap = ((int)(1.5 * rho_max * 4.0 / 3.0 * M_PI * rs3) + 32 + 7) & ~7;
    f->shell_cap = ((int)(1.5 * rho_max * 4.0 / 3.0 * M_PI * (rc3 - rs3) / pice_min) + 32 + 7) & ~7;
    if (f->cap_override > 0) f->core_cap = f->cap_override;
    f->cap = f->core_cap + f->shell_cap;
  }
  const size_t n = f->n;
  const bool fp64 = f->fp64;
  CK(dalloc(&f->d_reps, nrep));
  CK(cudaMemcpy(f->d_reps, f->reps_h.data(), sizeof(RepDev) * nrep, cudaMemcpyHostToDevice));
  CK(dalloc(&f->d_ljt, 1));
  CK(cudaMemcpy(f->d_ljt, &f->ljt_h, sizeof(LJTable), cudaMemcpyHostToDevice));
  std::vector<int> rep_of(n);
  for (int r = 0; r < nrep; ++r)
    for (int64_t i = f->rep_off[r]; i < f->rep_off[r + 1]; ++i) rep_of[i] = r;
  CK(dalloc(&f->d_rep_of, n));
  CK(cudaMemcpy(f->d_rep_of, rep_of.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
  CK(dalloc(&f->d_cell_of, n));
  CK(dalloc(&f->d_cell_count, (size_t)f->ncell_total));
  CK(dalloc(&f->d_cell_start, (size_t)f->ncell_total + 1));
  CK(dalloc(&f->d_cursor, (size_t)f->ncell_total));
  CK(dalloc(&f->d_tmp, n));
  CK(dalloc(&f->d_slot_atom, n));
  CK(dalloc(&f->d_atom_slot, n));
  CK(cudaMalloc(&f->d_pos4, n * (fp64 ? sizeof(double4) : sizeof(float4))));
  CK(dalloc(&f->d_meta, n));
  CK(dalloc(&f->d_nbr, (size_t)f->cap * f->stride));
  CK(dalloc(&f->d_count, n));
  if (f->is_rbl()) CK(dalloc(&f->d_count2, n));
  if (f->is_rbl() && f->rbl_table) {
    const std::vector<float> tab = rbl_erf_table();
    CK(dalloc(&f->d_erf_tab, tab.size()));
    CK(cudaMemcpy(f->d_erf_tab, tab.data(), sizeof(float) * tab.size(), cudaMemcpyHostToDevice));
  }
  if (f->nbr_type != "RBL" && f->num_cycles == 1) {
    // staged list build: segments of S x cells per (y, z) row, S sized so that a segment holds
    // about 224 atoms (one 256-thread pass) and its 9 x (S + 2) staged cells fill at most 60 %
    // of the shared buffer on average
    f->stage_cap = f->fp64 ? 2048 : 4096;
    std::vector<ListSeg> sg;
    for (int r = 0; r < nrep; ++r) {
      const RepDev& rp = f->reps_h[r];
      const double apc = std::max(1e-3, (double)(f->rep_off[r + 1] - f->rep_off[r]) / (double)rp.ncell);
      int S = (int)std::floor(224.0 / apc);
      S = std::min(S, (int)std::floor(0.6 * f->stage_cap / (9.0 * apc)) - 2);
      S = std::max(1, std::min(std::min(S, kSegMaxCells), rp.dims[0]));
      for (int z = 0; z < rp.dims[2]; ++z)
        for (int y = 0; y < rp.dims[1]; ++y)
          for (int x0 = 0; x0 < rp.dims[0]; x0 += S)
            sg.push_back(ListSeg{r, y, z, x0, std::min(x0 + S, rp.dims[0]), 0, 0, 0});
    }
    f->nsegs = (int)sg.size();
    CK(dalloc(&f->d_segs, sg.size()));
    CK(cudaMemcpy(f->d_segs, sg.data(), sizeof(ListSeg) * sg.size(), cudaMemcpyHostToDevice));
    const int bytes = f->stage_cap * (f->fp64 ? (int)sizeof(double4) : (int)sizeof(float4));
    CK(cudaFuncSetAttribute(f->fp64 ? (const void*)k_nlist_staged<double> : (const void*)k_nlist_staged<float>,
                            cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  }
  CK(dalloc(&f->d_maxcount, 2));
  CK(dalloc(&f->d_nbuilds, 1));
  CK(cudaMemset(f->d_nbuilds, 0, sizeof(unsigned long long)));
  CK(dalloc(&f->d_rebuild, (size_t)nrep + 1));
  CK(cudaMemset(f->d_rebuild, 0, sizeof(int) * (nrep + 1)));
  if (nrep > 1) {
    std::vector<int> cr(f->ncell_total);
    for (int r = 0; r < nrep; ++r)
      for (int c = 0; c < f->reps_h[r].ncell; ++c) cr[f->reps_h[r].cell_base + c] = r;
    CK(dalloc(&f->d_cell_rep, cr.size()));
    CK(cudaMemcpy(f->d_cell_rep, cr.data(), sizeof(int) * cr.size(), cudaMemcpyHostToDevice));
  }
  CK(dalloc(&f->d_block_sums, (size_t)(f->ncell_total + kScanBlock - 1) / kScanBlock + 1));
  if (f->skin > 0) CK(dalloc(&f->d_xref, 3 * n));
  CK(dalloc(&f->d_status, 1));
  CK(cudaMemset(f->d_status, 0, sizeof(uint32_t)));
  CK(dalloc(&f->d_step, 1));
  CK(cudaMemset(f->d_step, 0, sizeof(long long)));
  CK(dalloc(&f->d_lstep, 1));
  CK(cudaMemset(f->d_lstep, 0, sizeof(long long)));
  CK(dalloc(&f->d_eslot, 2 * n));
  CK(cudaMemset(f->d_eslot, 0, sizeof(double) * 2 * n));
  CK(dalloc(&f->d_esum, 32));
  CK(cudaMallocHost(&f->h_status, sizeof(uint32_t)));
  CK(cudaMallocHost(&f->h_maxcount, 2 * sizeof(int)));
  {
    // the k-space chain is short next to the near pass it overlaps: at the highest priority its
    // blocks take SMs as soon as near-pass blocks retire, so the join rarely waits
    int lo_prio = 0, hi_prio = 0;
    CK(cudaDeviceGetStreamPriorityRange(&lo_prio, &hi_prio));
    CK(cudaStreamCreateWithPriority(&f->side, cudaStreamNonBlocking, f->kspace_priority ? hi_prio : lo_prio));
  }
  CK(cudaEventCreateWithFlags(&f->ev_fork, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&f->ev_join, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&f->ev_tail, cudaEventDisableTiming));
  // host-side range checks: every device index derived from these arrays stays in bounds
  if (a->type) {
    std::vector<int> ty(n);
    CK(cudaMemcpy(ty.data(), a->type, sizeof(int) * n, cudaMemcpyDeviceToHost));
    for (int v : ty)
      if (v < 0 || v >= f->ntypes) {
        std::snprintf(g_last_error, sizeof g_last_error, "atom type %d outside [0, %d)", v, f->ntypes);
        return RBMD_ERR_ARG;
      }
  }
  for (int32_t v : f->hoh_h)
    if (v < 0 || v >= f->n) {
      std::snprintf(g_last_error, sizeof g_last_error, "water atom id %d outside [0, %d)", v, f->n);
      return RBMD_ERR_ARG;
    }
  // charges: sum q^2 for the self energy; compact list of charged atoms per replica
  f->sum_q2 = 0;
  std::vector<int> qidx;
  std::vector<int64_t> qoff(nrep + 1, 0);
  if (a->charge) {
    std::vector<double> q(n);
    CK(cudaMemcpy(q.data(), a->charge, sizeof(double) * n, cudaMemcpyDeviceToHost));
    for (double v : q) f->sum_q2 += v * v;
    for (int r = 0; r < nrep; ++r) {
      qoff[r] = (int64_t)qidx.size();
      for (int64_t i = f->rep_off[r]; i < f->rep_off[r + 1]; ++i)
        if (q[i] != 0.0) qidx.push_back((int)i);
    }
  }
  qoff[nrep] = (int64_t)qidx.size();
  f->nq = (int)qidx.size();
  // k-space
  if (f->is_rbe()) {
    CK(cudaMalloc(&f->d_frac, (size_t)std::max(1, f->nq) * (fp64 ? sizeof(Frac64) : sizeof(Frac32))));
    CK(dalloc(&f->d_far, 3 * (size_t)std::max(1, f->nq)));
    CK(dalloc(&f->d_qidx, (size_t)std::max(1, f->nq)));
    if (f->nq > 0)
      CK(cudaMemcpy(f->d_qidx, qidx.data(), sizeof(int) * f->nq, cudaMemcpyHostToDevice));
    const int recb = fp64 ? sizeof(KRec64) : sizeof(KRec32);
    if (f->coul_type == "EWALD") {
      // EWALD: the cube m in [-kmax, kmax]^3 \ {0} (ExecPointLocator::ExecuteOnKNeighbor,
      // ExecPointLocator.h:127-145) as a fixed sample set with weights e^{-k^2/4a} and S/P = 1.
      const int K = f->kmax;
      f->P = (2 * K + 1) * (2 * K + 1) * (2 * K + 1) - 1;
      for (int r = 0; r < nrep; ++r) {
        f->reps_h[r].P = f->P;
        f->reps_h[r].k_begin = r * f->P;
        f->reps_h[r].S = f->P;
      }
      CK(cudaMemcpy(f->d_reps, f->reps_h.data(), sizeof(RepDev) * nrep, cudaMemcpyHostToDevice));
    }
    f->Ptot = nrep * f->P;
    CK(cudaMalloc(&f->d_krec, (size_t)f->Ptot * recb));
    CK(cudaMemset(f->d_krec, 0, (size_t)f->Ptot * recb));
    CK(dalloc(&f->d_kvec, (size_t)3 * f->Ptot));
    CK(dalloc(&f->d_krep, (size_t)f->Ptot));
    {
      std::vector<int> krep(f->Ptot);
      for (int g = 0; g < f->Ptot; ++g) krep[g] = g / f->P;
      CK(cudaMemcpy(f->d_krep, krep.data(), sizeof(int) * f->Ptot, cudaMemcpyHostToDevice));
    }
    CK(dalloc(&f->d_rho, (size_t)f->Ptot));
    CK(dalloc(&f->d_ek, (size_t)f->Ptot));
    // structure-factor work items (replica, chunk, tile): a block has 32*kKL samples per warp and
    // at most 8 warps; chunks are sized for about four resident waves of blocks
    const int warps = std::min(8, (std::min(f->P, 8 * 32 * kKL) + 32 * kKL - 1) / (32 * kKL));
    f->rho_threads = 32 * warps;
    f->ktile = f->rho_threads * kKL;
    std::vector<RhoItem> items;
    std::vector<RhoRep> rr(nrep);
    const int ntiles = (f->P + f->ktile - 1) / f->ktile;
    const double target_blocks = 148.0 * (2048 / f->rho_threads) * 2.0;
    const double chunk_atoms = std::max(256.0, (double)std::max(1, f->nq) * ntiles / target_blocks);
    for (int r = 0; r < nrep; ++r) {
      const int Nr = (int)(qoff[r + 1] - qoff[r]);   // charged atoms of replica r
      const int nch = std::max(1, (int)std::lround(Nr / chunk_atoms));
      rr[r].item_base = (int)items.size();
      rr[r].ntiles = ntiles;
      rr[r].nchunks = nch;
      for (int c = 0; c < nch; ++c) {
        const int b = (int)qoff[r] + (int)((int64_t)Nr * c / nch);
        const int e = (int)qoff[r] + (int)((int64_t)Nr * (c + 1) / nch);
        for (int t = 0; t < ntiles; ++t) {
          RhoItem it;
          it.atom_begin = b;
          it.atom_end = e;
          it.k_first = f->reps_h[r].k_begin + t * f->ktile;
          it.k_count = std::min(f->ktile, f->P - t * f->ktile);
          items.push_back(it);
        }
      }
    }
    f->nitems = (int)items.size();
    CK(dalloc(&f->d_items, items.size()));
    CK(cudaMemcpy(f->d_items, items.data(), sizeof(RhoItem) * items.size(), cudaMemcpyHostToDevice));
    CK(dalloc(&f->d_rhorep, (size_t)nrep));
    CK(cudaMemcpy(f->d_rhorep, rr.data(), sizeof(RhoRep) * nrep, cudaMemcpyHostToDevice));
    CK(cudaMalloc(&f->d_partial, (size_t)f->nitems * f->ktile * 2 * (fp64 ? sizeof(double) : sizeof(float))));
    // shared-memory staging of k records in the force pass: the largest k range a 128-slot block
    // spans (slots keep replicas contiguous), capped by kStageBytes
    {
      int need = 0;
      for (int b0 = 0; b0 < f->nq; b0 += 128) {
        const int last = std::min(f->nq, b0 + 128) - 1;
        const int ra = rep_of[qidx[b0]], rb = rep_of[qidx[last]];
        need = std::max(need, (rb - ra + 1) * f->P);
      }
      const int cap_recs = kStageBytes / (int)recb;
      f->kstage = need <= cap_recs ? need : 0;
    }
    // sampler tables: G(m) = exp(-pi^2 m^2 / (alpha L^2)) / q(m) with q the rounding pmf of the
    // Gaussian proposal (Distribution_P / Distribution_q, rbmd/framework/model/RBEPSample.h:86-114)
    std::vector<SamplerRep> sr(nrep);
    std::vector<double> qtab;
    for (int r = 0; r < nrep; ++r) {
      const double* L = f->reps_h[r].box_d;
      SamplerRep& s = sr[r];
      s.qmax = 0;
      for (int d = 0; d < 3; ++d) {
        s.sigma[d] = std::sqrt(f->alpha / 2.0) * L[d] / M_PI;
        s.qmax = std::max(s.qmax, (int)std::ceil(14.0 * s.sigma[d]) + 8);
      }
      s.g_offset = (int)qtab.size();
      for (int d = 0; d < 3; ++d) {
        const double sc = std::sqrt(f->alpha * L[d] * L[d] / (M_PI * M_PI));
        const double c = M_PI * M_PI / (f->alpha * L[d] * L[d]);
        s.gmax[d] = 0.0;
        for (int m = 0; m <= s.qmax; ++m) {
          const double q = m == 0 ? std::erf(0.5 / sc)
                                  : (std::erf((0.5 + m) / sc) - std::erf((m - 0.5) / sc)) / 2.0;
          const double gv = q > 0 ? std::exp(-c * (double)m * (double)m) / q : INFINITY;
          qtab.push_back(gv);
          if (std::isfinite(gv)) s.gmax[d] = std::max(s.gmax[d], gv);
        }
      }
    }
    CK(dalloc(&f->d_srep, (size_t)nrep));
    CK(cudaMemcpy(f->d_srep, sr.data(), sizeof(SamplerRep) * nrep, cudaMemcpyHostToDevice));
    CK(dalloc(&f->d_qtab, qtab.size()));
    CK(cudaMemcpy(f->d_qtab, qtab.data(), sizeof(double) * qtab.size(), cudaMemcpyHostToDevice));
    if (f->coul_type == "RBE" && f->proposal != "gauss") {
      rbmd_status st = build_proposal_tables(f, qoff);
      if (st) return st;
    }
    if (f->coul_type == "EWALD") {
      // fixed cube sample set with Gaussian weights
      std::vector<int> m;
      std::vector<double> w;
      for (int r = 0; r < nrep; ++r) {
        const double* L = f->reps_h[r].box_d;
        const int K = f->kmax;
        for (int i = -K; i <= K; ++i)
          for (int j = -K; j <= K; ++j)
            for (int k = -K; k <= K; ++k) {
              if (i == 0 && j == 0 && k == 0) continue;
              m.push_back(i); m.push_back(j); m.push_back(k);
              const double kx = 2 * M_PI * i / L[0], ky = 2 * M_PI * j / L[1], kz = 2 * M_PI * k / L[2];
              w.push_back(std::exp(-(kx * kx + ky * ky + kz * kz) / (4 * f->alpha)));
            }
      }
      rbmd_status s2 = upload_ksamples(f, m.data());
      if (s2) return s2;
      CK(dalloc(&f->d_weights, w.size()));
      CK(cudaMemcpy(f->d_weights, w.data(), sizeof(double) * w.size(), cudaMemcpyHostToDevice));
    }
  }
  // MD chunks
  {
    std::vector<MdChunk> ch;
    std::vector<int> crb(nrep + 1);
    for (int r = 0; r < nrep; ++r) {
      crb[r] = (int)ch.size();
      for (int64_t b = f->rep_off[r]; b < f->rep_off[r + 1]; b += kMdChunk) {
        MdChunk c;
        c.begin = (int)b;
        c.end = (int)std::min<int64_t>(b + kMdChunk, f->rep_off[r + 1]);
        c.rep = r;
        c.pad = 0;
        ch.push_back(c);
      }
    }
    crb[nrep] = (int)ch.size();
    f->nchunks = (int)ch.size();
    CK(dalloc(&f->d_chunks, ch.size()));
    CK(cudaMemcpy(f->d_chunks, ch.data(), sizeof(MdChunk) * ch.size(), cudaMemcpyHostToDevice));
    CK(dalloc(&f->d_chunk_rep_begin, (size_t)nrep + 1));
    CK(cudaMemcpy(f->d_chunk_rep_begin, crb.data(), sizeof(int) * (nrep + 1), cudaMemcpyHostToDevice));
    CK(dalloc(&f->d_ke_partial, ch.size()));
    if (f->is_rbl()) CK(dalloc(&f->d_mean_partial, 3 * ch.size()));
    CK(dalloc(&f->d_ke, (size_t)nrep));
    CK(dalloc(&f->d_T, (size_t)nrep));
    CK(dalloc(&f->d_lambda, (size_t)nrep));
    CK(dalloc(&f->d_xi, (size_t)nrep));
    CK(cudaMemset(f->d_xi, 0, sizeof(double) * nrep));
    CK(cudaMemset(f->d_ke, 0, sizeof(double) * nrep));
    CK(cudaMemset(f->d_T, 0, sizeof(double) * nrep));
    std::vector<double> ones(nrep, 1.0);
    CK(cudaMemcpy(f->d_lambda, ones.data(), sizeof(double) * nrep, cudaMemcpyHostToDevice));
    if (f->shake == "true" && f->n_mol > 0) {
      CK(dalloc(&f->d_xold, 3 * n));
      CK(dalloc(&f->d_vold, 3 * n));
    }
  }
  // EAM
  if (f->is_eam()) {
    auto up = [&](const std::vector<float>& s, float4** d) -> rbmd_status {
      const size_t rows = s.size() / 7;
      std::vector<float4> v(2 * rows);
      for (size_t m = 0; m < rows; ++m) {
        v[2 * m] = make_float4(s[7 * m], s[7 * m + 1], s[7 * m + 2], s[7 * m + 3]);
        v[2 * m + 1] = make_float4(s[7 * m + 4], s[7 * m + 5], s[7 * m + 6], 0.f);
      }
      CK(dalloc(d, v.size()));
      CK(cudaMemcpy(*d, v.data(), sizeof(float4) * v.size(), cudaMemcpyHostToDevice));
      return RBMD_OK;
    };
    rbmd_status s1 = up(f->eam_h.frho, &f->d_frho);
    if (s1) return s1;
    s1 = up(f->eam_h.rhor, &f->d_rhor);
    if (s1) return s1;
    s1 = up(f->eam_h.z2r, &f->d_z2r);
    if (s1) return s1;
    CK(cudaMalloc(&f->d_fp, n * (fp64 ? sizeof(double) : sizeof(float))));
    CK(dalloc(&f->d_emb, n));
    CK(dalloc(&f->d_epair, n));
  }
  // water
  if (f->n_mol > 0) {
    CK(dalloc(&f->d_hoh, (size_t)3 * f->n_mol));
    CK(cudaMemcpy(f->d_hoh, f->hoh_h.data(), sizeof(int) * 3 * f->n_mol, cudaMemcpyHostToDevice));
    CK(dalloc(&f->d_ebond, (size_t)f->n_mol));
    CK(dalloc(&f->d_eangle, (size_t)f->n_mol));
    CK(dalloc(&f->d_ewcoul, (size_t)f->n_mol));
  }
  {
    rbmd_status st = upload_topology(f);
    if (st) return st;
  }
  CK(dalloc(&f->d_host32, (size_t)3 * f->n));
  f->bound = true;
  f->list_valid = false;
  f->step_count = 0;
  f->pending_scale = false;
  return RBMD_OK;
}

rbmd_status rbmd_force_set_ksamples(rbmd_force* f, const int32_t* m_xyz, int32_t P) {
  if (f) drop_graphs(f);
  if (!f) return RBMD_ERR_ARG;
  if (!m_xyz || P == 0) {
    f->injected = false;
    return RBMD_OK;
  }
  if (!f->bound || !f->is_rbe() || P != f->P || f->coul_type != "RBE") return RBMD_ERR_ARG;
  return upload_ksamples(f, m_xyz);
}

rbmd_status rbmd_force_set_kweights(rbmd_force* f, const double* w_host) {
  if (f) drop_graphs(f);
  if (!f || !f->bound || !f->is_rbe()) return RBMD_ERR_ARG;
  if (!w_host) { dfree(f->d_weights); return RBMD_OK; }
  if (!f->d_weights) CK(dalloc(&f->d_weights, (size_t)f->Ptot));
  CK(cudaMemcpy(f->d_weights, w_host, sizeof(double) * f->Ptot, cudaMemcpyHostToDevice));
  return RBMD_OK;
}

rbmd_status rbmd_force_get_ksamples(rbmd_force* f, int32_t* m_xyz, int32_t P) {
  if (!f || !m_xyz || !f->bound || !f->is_rbe() || P != f->P) return RBMD_ERR_ARG;
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(m_xyz, f->d_kvec, sizeof(int) * 3 * f->Ptot, cudaMemcpyDeviceToHost));
  return RBMD_OK;
}

rbmd_status rbmd_force_sample_k(rbmd_force* f, int64_t step, int32_t* m_xyz, int32_t P) {
  if (!f || !f->bound || !f->is_rbe() || P != f->P || f->coul_type != "RBE") return RBMD_ERR_ARG;
  const int recb = f->fp64 ? sizeof(KRec64) : sizeof(KRec32);
  f->presampled = false;   // overwrites the k-set buffers
  if (f->proposal != "gauss")
    launch_prop_sample(f, nullptr, step, recb);
  else
    k_sample<kSamplerD><<<f->nrep, 256>>>(f->nrep, f->d_srep, f->d_qtab, f->d_reps, f->seed, step, nullptr,
                                           f->d_kvec, f->d_krec, recb, f->d_krep, f->d_status);
  CK(cudaGetLastError());
  CK(cudaDeviceSynchronize());
  if (m_xyz) CK(cudaMemcpy(m_xyz, f->d_kvec, sizeof(int) * 3 * f->Ptot, cudaMemcpyDeviceToHost));
  return RBMD_OK;
}

rbmd_status rbmd_force_autotune(rbmd_force* f, void* stream, int32_t* list_lanes, int32_t* force_lanes) {
  if (f) drop_graphs(f);
  if (!f) return RBMD_ERR_ARG;
  if (!f->bound) return RBMD_ERR_STATE;
  cudaStream_t s = (cudaStream_t)stream;
  f->launches = 0;
  launch_compute_any(f, s);            // current list and caches
  bool redo = false;
  rbmd_status st = check_overflow(f, s, &redo);
  if (st) return st;
  if (redo) {
    launch_compute_any(f, s);
    st = check_overflow(f, s, &redo);
    if (st) return st;
  }
  st = f->fp64 ? autotune_impl<double>(f, s) : autotune_impl<float>(f, s);
  if (st) return st;
  launch_compute_any(f, s);            // leave forces of the chosen configuration
  st = check_overflow(f, s, &redo);
  if (st) return st;
  if (list_lanes) *list_lanes = f->tpa_list;
  if (force_lanes) *force_lanes = f->near_lanes > 1 ? -f->near_lanes : f->tpa_near;
  return RBMD_OK;
}

rbmd_status rbmd_force_compute(rbmd_force* f, void* stream) {
  if (!f) return RBMD_ERR_ARG;
  if (!f->bound) return RBMD_ERR_STATE;
  cudaStream_t s = (cudaStream_t)stream;
  if (f->autotune && !f->tuned) return rbmd_force_autotune(f, stream, nullptr, nullptr);
  for (int attempt = 0; attempt < 4; ++attempt) {
    f->launches = 0;
    launch_compute_any(f, s);
    CK(cudaGetLastError());
    bool redo = false;
    rbmd_status st = check_overflow(f, s, &redo);
    if (st) return st;
    if (!redo) return RBMD_OK;
  }
  return RBMD_ERR_DEVICE;
}

rbmd_status rbmd_force_compute_host(rbmd_force* f, const double* pos_host, double* force_host,
                                    void* stream) {
  if (!f || !pos_host || !force_host) return RBMD_ERR_ARG;
  if (!f->bound) return RBMD_ERR_STATE;
  cudaStream_t s = (cudaStream_t)stream;
  CK(cudaMemcpyAsync(f->at.pos, pos_host, sizeof(double) * 3 * f->n, cudaMemcpyHostToDevice, s));
  for (int attempt = 0; attempt < 4; ++attempt) {
    f->launches = 0;
    launch_compute_any(f, s);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(force_host, f->at.force, sizeof(double) * 3 * f->n, cudaMemcpyDeviceToHost, s));
    bool redo = false;
    rbmd_status st = check_overflow(f, s, &redo);
    if (st) return st;
    if (!redo) return RBMD_OK;
  }
  return RBMD_ERR_DEVICE;
}

rbmd_status rbmd_force_compute_host_f32(rbmd_force* f, const float* pos_host, float* force_host, void* stream) {
  if (!f || !pos_host || !force_host) return RBMD_ERR_ARG;
  if (!f->bound) return RBMD_ERR_STATE;
  cudaStream_t s = (cudaStream_t)stream;
  const long long m = 3LL * f->n;
  const int grid = (int)std::min<long long>((m + 255) / 256, 8LL * f->num_sms);
  CK(cudaMemcpyAsync(f->d_host32, pos_host, sizeof(float) * m, cudaMemcpyHostToDevice, s));
  k_f32_to_f64<<<grid, 256, 0, s>>>(m, f->d_host32, f->at.pos);
  for (int attempt = 0; attempt < 4; ++attempt) {
    f->launches = 1;
    launch_compute_any(f, s);
    k_f64_to_f32<<<grid, 256, 0, s>>>(m, f->at.force, f->d_host32);
    f->launches++;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(force_host, f->d_host32, sizeof(float) * m, cudaMemcpyDeviceToHost, s));
    bool redo = false;
    rbmd_status st = check_overflow(f, s, &redo);
    if (st) return st;
    if (!redo) return RBMD_OK;
  }
  return RBMD_ERR_DEVICE;
}

rbmd_status rbmd_force_step(rbmd_force* f, int32_t n_steps, void* stream) {
  if (!f || n_steps < 0) return RBMD_ERR_ARG;
  if (!f->bound) return RBMD_ERR_STATE;
  if (!f->at.vel || !f->at.mass) return RBMD_ERR_STATE;
  cudaStream_t s = (cudaStream_t)stream;
  const size_t n = f->n;
  if (!f->d_snap) CK(dalloc(&f->d_snap, 9 * n));
  if (f->at.image && !f->d_snap_img) CK(dalloc(&f->d_snap_img, 3 * n));
  const long long step0 = f->step_count;
  const bool pend0 = f->pending_scale;
  for (int attempt = 0; attempt < 4; ++attempt) {
    CK(cudaMemcpyAsync(f->d_snap, f->at.pos, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(f->d_snap + 3 * n, f->at.vel, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(f->d_snap + 6 * n, f->at.force, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice, s));
    if (f->at.image)
      CK(cudaMemcpyAsync(f->d_snap_img, f->at.image, sizeof(int) * 3 * n, cudaMemcpyDeviceToDevice, s));
    f->launches = 0;
    CK(cudaMemcpyAsync(f->d_step, &f->step_count, sizeof(long long), cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));
    f->in_step = true;
    rbmd_status gs = f->fp64 ? run_steps<double>(f, n_steps, s) : run_steps<float>(f, n_steps, s);
    f->in_step = false;
    if (gs) return gs;
    CK(cudaGetLastError());
    bool redo = false;
    rbmd_status st = check_overflow(f, s, &redo);
    if (st) return st;
    if (!redo) {
      if (n_steps > 0) f->launches /= n_steps;
      return RBMD_OK;
    }
    // replay from the snapshot with the grown list (the sampler is keyed by the step counter)
    CK(cudaMemcpyAsync(f->at.pos, f->d_snap, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(f->at.vel, f->d_snap + 3 * n, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(f->at.force, f->d_snap + 6 * n, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice, s));
    if (f->at.image)
      CK(cudaMemcpyAsync(f->at.image, f->d_snap_img, sizeof(int) * 3 * n, cudaMemcpyDeviceToDevice, s));
    f->step_count = step0;
    f->pending_scale = pend0;
  }
  return RBMD_ERR_DEVICE;
}

// Apply a deferred thermostat rescale so that the bound velocities are current.
rbmd_status rbmd_force_sync_velocities(rbmd_force* f, void* stream) {
  if (!f || !f->bound) return RBMD_ERR_STATE;
  if (f->pending_scale) {
    k_scale_vel<<<(f->n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        f->n, f->nrep > 1 ? f->d_rep_of : nullptr, f->d_lambda, f->at.vel);
    CK(cudaGetLastError());
    f->pending_scale = false;
  }
  return RBMD_OK;
}

rbmd_status rbmd_force_energy(rbmd_force* f, rbmd_energy* out, void* stream) {
  if (!f || !out) return RBMD_ERR_ARG;
  if (!f->bound) return RBMD_ERR_STATE;
  cudaStream_t s = (cudaStream_t)stream;
  std::memset(out, 0, sizeof *out);
  CK(cudaMemsetAsync(f->d_esum, 0, sizeof(double) * 32, s));
  if (!f->is_eam()) {
    k_sum<<<1, 1024, 0, s>>>(f->n, f->d_eslot, 2, 0, f->d_esum + 0);
    k_sum<<<1, 1024, 0, s>>>(f->n, f->d_eslot, 2, 1, f->d_esum + 1);
  } else {
    k_sum<<<1, 1024, 0, s>>>(f->n, f->d_emb, 1, 0, f->d_esum + 4);
    k_sum<<<1, 1024, 0, s>>>(f->n, f->d_epair, 1, 0, f->d_esum + 5);
  }
  if (f->is_rbe()) k_sum<<<1, 1024, 0, s>>>(f->Ptot, f->d_ek, 1, 0, f->d_esum + 2);
  if (f->topo && f->is_cvff()) {
    if (f->topo_nb) k_sum<<<1, 1024, 0, s>>>(f->topo_nb, f->d_eterm, 1, 0, f->d_esum + 6);
    if (f->topo_na) k_sum<<<1, 1024, 0, s>>>(f->topo_na, f->d_eterm + f->topo_nb, 1, 0, f->d_esum + 7);
    if (f->topo_nd)
      k_sum<<<1, 1024, 0, s>>>(f->topo_nd, f->d_eterm + f->topo_nb + f->topo_na, 1, 0, f->d_esum + 10);
    k_sum<<<1, 1024, 0, s>>>(f->n, f->d_esc, 1, 0, f->d_esum + 11);
  } else if (f->n_mol > 0 && f->is_cvff()) {
    k_sum<<<1, 1024, 0, s>>>((int)f->n_mol, f->d_ebond, 1, 0, f->d_esum + 6);
    k_sum<<<1, 1024, 0, s>>>((int)f->n_mol, f->d_eangle, 1, 0, f->d_esum + 7);
    k_sum<<<1, 1024, 0, s>>>((int)f->n_mol, f->d_ewcoul, 1, 0, f->d_esum + 11);
  }
  k_sum<<<1, 1024, 0, s>>>(f->nrep, f->d_ke, 1, 0, f->d_esum + 8);
  k_sum<<<1, 1024, 0, s>>>(f->nrep, f->d_T, 1, 0, f->d_esum + 9);
  CK(cudaGetLastError());
  double h[16];
  CK(cudaMemcpyAsync(h, f->d_esum, sizeof(double) * 16, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  out->lj = h[0];
  out->coul_real = h[1];
  out->coul_kspace = h[2];
  out->coul_self = f->is_rbe() ? -std::sqrt(f->alpha / M_PI) * f->sum_q2 * f->u.qqr2e : 0.0;
  out->eam_embed = h[4];
  out->eam_pair = h[5];
  out->bond = h[6];
  out->angle = h[7];
  out->kinetic = h[8];
  out->temperature = h[9] / f->nrep;
  out->dihedral = h[10];
  out->coul_special = h[11];
  return RBMD_OK;
}

rbmd_status rbmd_force_status(rbmd_force* f, uint32_t* flags, int32_t clear, void* stream) {
  if (!f || !flags) return RBMD_ERR_ARG;
  if (!f->bound) { *flags = 0; return RBMD_OK; }
  cudaStream_t s = (cudaStream_t)stream;
  CK(cudaMemcpyAsync(f->h_status, f->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  *flags = *f->h_status;
  if (clear) CK(cudaMemsetAsync(f->d_status, 0, sizeof(uint32_t), s));
  CK(cudaStreamSynchronize(s));
  return RBMD_OK;
}

rbmd_status rbmd_force_get_neighbors(rbmd_force* f, int32_t* counts, int32_t* ids, int64_t cap) {
  if (!f || !counts || !ids || cap < 0) return RBMD_ERR_ARG;
  if (!f->bound) return RBMD_ERR_STATE;
  CK(cudaDeviceSynchronize());
  const size_t n = f->n;
  std::vector<int> cnt(n), cnt2(n, 0), slot_atom(n), nbr((size_t)f->cap * f->stride);
  CK(cudaMemcpy(cnt.data(), f->d_count, sizeof(int) * n, cudaMemcpyDeviceToHost));
  if (f->is_rbl()) CK(cudaMemcpy(cnt2.data(), f->d_count2, sizeof(int) * n, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(slot_atom.data(), f->d_slot_atom, sizeof(int) * n, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(nbr.data(), f->d_nbr, sizeof(int) * nbr.size(), cudaMemcpyDeviceToHost));
  bool too_small = false;
  // RBL: the core pairs followed by the kept shell pairs, each in traversal order
  const int cap_a = f->is_rbl() ? f->core_cap : f->cap;
  for (size_t i = 0; i < n; ++i) {
    const int id = slot_atom[i];
    const int ma = std::min<int>(cnt[i], cap_a);
    const int mb = f->is_rbl() ? std::min<int>(cnt2[i], f->shell_cap) : 0;
    counts[id] = ma + mb;
    if (ma + mb > cap) too_small = true;
    for (int p = 0; p < ma + mb && p < cap; ++p) {
      const int row = p < ma ? p : cap_a + (p - ma);
      ids[(size_t)id * cap + p] = slot_atom[nbr[(size_t)row * f->stride + i] >> kShiftBits];
    }
  }
  return too_small ? RBMD_ERR_ARG : RBMD_OK;
}

rbmd_status rbmd_force_get_rbl(rbmd_force* f, int32_t* ncore, int32_t* nshell, int64_t* sizes) {
  if (!f || !sizes) return RBMD_ERR_ARG;
  if (!f->bound || !f->is_rbl()) return RBMD_ERR_STATE;
  CK(cudaDeviceSynchronize());
  const size_t n = f->n;
  std::vector<int> a(n), b(n), slot_atom(n);
  CK(cudaMemcpy(a.data(), f->d_count, sizeof(int) * n, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(b.data(), f->d_count2, sizeof(int) * n, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(slot_atom.data(), f->d_slot_atom, sizeof(int) * n, cudaMemcpyDeviceToHost));
  for (size_t i = 0; i < n; ++i) {
    if (ncore) ncore[slot_atom[i]] = a[i];
    if (nshell) nshell[slot_atom[i]] = b[i];
  }
  sizes[0] = f->rbl_sizes_h[0];
  sizes[1] = f->rbl_sizes_h[1];
  sizes[2] = f->rbl_sizes_h[2];
  sizes[3] = f->core_cap;
  sizes[4] = f->shell_cap;
  return RBMD_OK;
}

rbmd_status rbmd_force_train_proposal(rbmd_force* f, const rbmd_train_opts* o, rbmd_train_report* rep,
                                      void* stream) {
  if (f) drop_graphs(f);
  if (!f || !o) return RBMD_ERR_ARG;
  if (!f->bound || f->proposal != "learned" || !f->d_prep) return RBMD_ERR_STATE;
  if (o->n_snapshots < 1 || o->k_per_snapshot < 256 || o->iterations < 1 || o->steps_between < 0 ||
      !(o->learning_rate > 0))
    return RBMD_ERR_ARG;
  const auto t0 = std::chrono::steady_clock::now();
  cudaStream_t s = (cudaStream_t)stream;
  const int S = o->n_snapshots, K = o->k_per_snapshot, nq0 = f->prep_h[0].nq;
  if (nq0 < 1) return RBMD_ERR_STATE;
  const int nch = (nq0 + kTrainChunk - 1) / kTrainChunk;
  TrainScratch ts;
  int *kv = nullptr, *krec = nullptr, *krep = nullptr, *kbin = nullptr;
  double *kw = nullptr, *ak = nullptr, *loss = nullptr;
  double2* rho = nullptr;
  float *partial = nullptr, *cbin = nullptr, *spec = nullptr, *wbinf = nullptr, *X = nullptr, *gpart = nullptr,
        *grad = nullptr, *am = nullptr, *av = nullptr;
  Frac32* frac = nullptr;
  RepDev* rep1 = nullptr;
  CK(ts.get(&kv, 3 * (size_t)K));
  CK(ts.get(&krec, 3 * (size_t)K));
  CK(ts.get(&krep, (size_t)K));
  CK(ts.get(&kbin, (size_t)K));
  CK(ts.get(&kw, (size_t)K));
  CK(ts.get(&ak, (size_t)K));
  CK(ts.get(&rho, (size_t)K));
  CK(ts.get(&partial, 2 * (size_t)nch * K));
  CK(ts.get(&cbin, (size_t)S * kPropBins));
  CK(ts.get(&spec, (size_t)S * kPropBands));
  CK(ts.get(&wbinf, (size_t)S * kPropBins));
  CK(ts.get(&X, (size_t)S * kPropBins * kMlpIn));
  CK(ts.get(&loss, (size_t)S));
  CK(ts.get(&gpart, (size_t)S * kMlpNParam));
  CK(ts.get(&grad, (size_t)kMlpNParam));
  CK(ts.get(&am, (size_t)kMlpNParam));
  CK(ts.get(&av, (size_t)kMlpNParam));
  CK(ts.get(&frac, (size_t)nq0));
  CK(ts.get(&rep1, 1));
  {
    RepDev r1 = f->reps_h[0];
    r1.P = K;
    r1.k_begin = 0;
    CK(cudaMemcpy(rep1, &r1, sizeof r1, cudaMemcpyHostToDevice));
  }
  const int* rep_of = f->nrep > 1 ? f->d_rep_of : nullptr;
  // ---- data: per snapshot, K draws from p, exact rho_k, per-sample force norms, bins ----
  for (int sn = 0; sn < S; ++sn) {
    if (o->steps_between > 0) {
      rbmd_status st = rbmd_force_step(f, o->steps_between, stream);
      if (st) return st;
    }
    k_frac<float><<<(nq0 + 255) / 256, 256, 0, s>>>(nq0, f->d_qidx, f->at.pos, f->at.charge, rep_of, f->d_reps,
                                                     frac);
    k_prop_sample<<<1, kSampThreads, f->prop_stage_bytes, s>>>(1, rep1, f->d_prep, f->d_cdf, nullptr, f->d_wbin, o->seed,
                                    (1LL << 40) + sn, nullptr, 4096, kv, krec, 12, krep, kw, f->d_status);
    const dim3 grid((K + 255) / 256, nch);
    for (int pass = 0; pass < 2; ++pass) {
      k_train_pass<<<grid, 256, 0, s>>>(pass, K, nq0, frac, kv, rho, partial);
      k_train_finish<<<(K + 255) / 256, 256, 0, s>>>(pass, K, nch, f->d_prep, kv, partial, rho, ak, kbin);
    }
    k_train_bins<<<1, kPropBins, 0, s>>>(K, nq0, kbin, rho, ak, cbin + (size_t)sn * kPropBins,
                                         spec + (size_t)sn * kPropBands);
    CK(cudaGetLastError());
  }
  return train_fit(f, o, rep, s, t0, S, cbin, spec, wbinf, X, loss, gpart, grad, am, av);
}

rbmd_status rbmd_force_proposal_params(rbmd_force* f, float* get_host, const float* set_host) {
  if (f && set_host) drop_graphs(f);
  if (!f || (!get_host && !set_host)) return RBMD_ERR_ARG;
  if (!f->bound || !f->d_mlp) return RBMD_ERR_STATE;
  if (set_host) {
    CK(cudaMemcpy(f->d_mlp, set_host, sizeof(float) * kMlpNParam, cudaMemcpyHostToDevice));
    CK(mlp_prepare(f->d_mlp, f->d_mlp_t, nullptr));
    CK(cudaDeviceSynchronize());
    f->prop_trained = true;
    f->presampled = false;
  }
  if (get_host) CK(cudaMemcpy(get_host, f->d_mlp, sizeof(float) * kMlpNParam, cudaMemcpyDeviceToHost));
  return RBMD_OK;
}

rbmd_status rbmd_force_get_far(rbmd_force* f, double* far_host) {
  if (!f || !far_host) return RBMD_ERR_ARG;
  if (!f->bound || !f->is_rbe()) return RBMD_ERR_STATE;
  CK(cudaDeviceSynchronize());
  std::memset(far_host, 0, sizeof(double) * 3 * (size_t)f->n);
  if (f->nq == 0) return RBMD_OK;
  std::vector<double> far(3 * (size_t)f->nq);
  std::vector<int> q(f->nq);
  CK(cudaMemcpy(far.data(), f->d_far, sizeof(double) * far.size(), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(q.data(), f->d_qidx, sizeof(int) * q.size(), cudaMemcpyDeviceToHost));
  for (int c = 0; c < f->nq; ++c)
    for (int d = 0; d < 3; ++d) far_host[3 * (size_t)q[c] + d] = far[3 * (size_t)c + d];
  return RBMD_OK;
}

rbmd_status rbmd_force_get_rhok(rbmd_force* f, double* rho, int32_t P) {
  if (!f || !rho || !f->bound || !f->is_rbe() || P != f->P) return RBMD_ERR_ARG;
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(rho, f->d_rho, sizeof(double2) * f->Ptot, cudaMemcpyDeviceToHost));
  return RBMD_OK;
}

rbmd_status rbmd_force_profile(rbmd_force* f, int32_t enable) {
  if (!f) return RBMD_ERR_ARG;
  f->prof_on = enable != 0;
  for (int i = 0; i < 8; ++i) { f->phase_ms[i] = 0; f->phase_n[i] = 0; }
  return RBMD_OK;
}

rbmd_status rbmd_force_phase_ms(rbmd_force* f, double* ms, int64_t* counts, int32_t n) {
  if (!f || !ms || n < 1) return RBMD_ERR_ARG;
  for (int i = 0; i < n && i < 8; ++i) {
    ms[i] = f->phase_ms[i];
    if (counts) counts[i] = f->phase_n[i];
  }
  return RBMD_OK;
}

rbmd_status rbmd_force_list_builds(rbmd_force* f, int64_t* builds) {
  if (!f || !builds) return RBMD_ERR_ARG;
  if (!f->bound) { *builds = 0; return RBMD_OK; }
  unsigned long long v = 0;
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(&v, f->d_nbuilds, sizeof v, cudaMemcpyDeviceToHost));
  *builds = (int64_t)v;
  return RBMD_OK;
}

rbmd_status rbmd_force_launch_count(rbmd_force* f, int32_t* k) {
  if (!f || !k) return RBMD_ERR_ARG;
  *k = f->launches;
  return RBMD_OK;
}

void rbmd_force_destroy(rbmd_force* f) {
  if (!f) return;
  if (f->bound) cudaDeviceSynchronize();
  free_all(f);
  delete f;
}

}  // extern "C"
