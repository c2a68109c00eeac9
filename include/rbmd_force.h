/*
 * rbmd_force.h -- C ABI of the B200 (sm_100a) per-timestep force path of RBMD.
 *
 * The reference selects its force path by string dispatch inside
 * ExecutionNVT::ComputeAllForce (rbmd/framework/run/ExecutionNVT.cpp:185-222), keyed by
 * force_field.type, neighbor.type and coulomb.type, and the HIP tree exposes the same path
 * as `class Force { virtual void Init(); virtual void Execute() = 0; }`
 * (rbmd-gpu-clone/rbmd-gpu/src/force/include/force.h:8-25).  This header replaces both with
 * plain C entry points: no C++ types, no CUDA types (streams are passed as `void*` holding a
 * cudaStream_t), plain pointers and sizes.
 *
 * Ownership: the caller owns the atom arrays (device pointers, caller's atom order).  The
 * library owns cells, neighbour lists, k-space buffers and its workspace.  Every call returns
 * an rbmd_status; device-side failures are reported through a status word
 * (rbmd_force_status) and never terminate the process (the reference calls exit(0) from
 * console::Error, rbmd/framework/Logging.h:45-51).
 */
#ifndef RBMD_FORCE_H
#define RBMD_FORCE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define RBMD_API __attribute__((visibility("default")))
#else
#define RBMD_API
#endif

typedef int32_t rbmd_status;

/* host-side return codes */
#define RBMD_OK                 0
#define RBMD_ERR_ARG            1   /* bad argument (null pointer, size, unknown key value) */
#define RBMD_ERR_CONFIG         2   /* JSON text could not be parsed or misses a required key */
#define RBMD_ERR_CUDA           3   /* a CUDA runtime call failed */
#define RBMD_ERR_STATE          4   /* call order violated (e.g. compute before bind) */
#define RBMD_ERR_DEVICE         5   /* the device status word holds an error bit */
#define RBMD_ERR_FILE           6   /* potential / data file unreadable */

/* device status word bits (rbmd_force_status) */
#define RBMD_FLAG_LIST_OVERFLOW   0x01u  /* an atom had more neighbours than the list capacity */
#define RBMD_FLAG_CELL_OVERFLOW   0x02u  /* a cell held more atoms than the cell sort supports */
#define RBMD_FLAG_SHAKE_NOCONV    0x04u  /* SHAKE hit its iteration cap before |dlambda|<tol */
#define RBMD_FLAG_NONFINITE       0x08u  /* a NaN/Inf force or position was produced */
#define RBMD_FLAG_OUT_OF_BOX      0x10u  /* an atom moved more than one box length in a step */
#define RBMD_FLAG_SAMPLER         0x20u  /* the k-sampler ran out of pre-drawn proposals */
#define RBMD_FLAG_SHAKE_SINGULAR  0x40u  /* |det| of a SHAKE/RATTLE matrix fell below 1e-4 */

typedef struct rbmd_force rbmd_force;

/* Orthorhombic periodic box of one replica: [lo, hi) per axis, as the LAMMPS header
 * "xlo xhi" lines give it (rbmd/framework/InitCondition/ModelFileInitCondition.cpp:176-221). */
typedef struct {
  double lo[3];
  double hi[3];
} rbmd_box;

/* Device atom arrays, caller atom order.  Replica r owns atoms
 * [replica_offsets[r], replica_offsets[r+1]).  Optional pointers may be NULL. */
typedef struct {
  int64_t n_atoms;
  int32_t n_replicas;
  const int64_t* replica_offsets; /* HOST array, n_replicas+1 entries; NULL when n_replicas==1 */
  double* pos;                    /* [n_atoms*3] x,y,z interleaved, FP64 master positions   */
  double* vel;                    /* [n_atoms*3] FP64 velocities (step API only; may be NULL)*/
  double* force;                  /* [n_atoms*3] output, FP64                                */
  const double* mass;             /* [n_atoms] per-atom mass (step API only; may be NULL)    */
  const double* charge;           /* [n_atoms] charge in e (NULL = all zero)                 */
  const int32_t* type;            /* [n_atoms] 0-based atom type (NULL = all type 0)         */
  const int32_t* molecule;        /* [n_atoms] 0-based molecule id (NULL = atom index)       */
  int32_t* image;                 /* [n_atoms*3] periodic image flags (NULL = not tracked)   */
} rbmd_atoms_dev;

/* Energies of the last compute (device sums, FP64).  Units follow the configured unit set. */
typedef struct {
  double lj;           /* 12-6 pair energy                                   */
  double coul_real;    /* erfc real-space Coulomb (x qqr2e)                   */
  double coul_kspace;  /* k-space estimate of the Ewald reciprocal energy     */
  double coul_self;    /* -sqrt(alpha/pi) * sum q^2 (x qqr2e)                 */
  double eam_embed;    /* sum F(rho_i)                                        */
  double eam_pair;     /* 1/2 sum phi(r_ij)                                   */
  double bond;         /* harmonic bonds                                      */
  double angle;        /* harmonic angles                                     */
  double kinetic;      /* 1/2 sum m v^2 * mvv2e (step API)                     */
  double temperature;  /* as ExecutionNVT::ComputeTempe (step API)            */
  double dihedral;     /* harmonic dihedrals (rbmd_force_set_topology)        */
  double coul_special; /* intramolecular Coulomb correction (set_topology)    */
} rbmd_energy;

/* Create a force path from RBMD's JSON configuration text (the same "hyper_parameters",
 * "execution" and "init_configuration" keys as rbmd/framework/hyperparameters/*.cpp and
 * rbmd/framework/run/ExecutionMD.cpp:144-153 read; optional extra keys: neighbor.skin,
 * coulomb.seed, precision ("fp32"|"fp64")).  `boxes` holds one box per replica.
 * Replaces: ExecutionNVT constructor + InitParameters + SetForceFunction
 * (rbmd/framework/run/ExecutionNVT.cpp:52-58,789-833). */
RBMD_API rbmd_status rbmd_force_create(const char* json_text, int32_t n_replicas, const rbmd_box* boxes,
                              rbmd_force** out);

/* Per-type 12-6 parameters, the "Pair Coeffs" section of the data file
 * (rbmd/framework/InitCondition/ModelFileInitCondition.cpp:297-323). */
RBMD_API rbmd_status rbmd_force_set_pair_coeffs(rbmd_force* f, int32_t n_types, const double* epsilon,
                                       const double* sigma);

/* EAM: read a funcfl potential file and build the 7-coefficient splines exactly as
 * ExecutionNVT::ReadPotentialFile/file2array/array2spline do
 * (rbmd/framework/run/ExecutionNVT.cpp:903-1107).  Called by create when
 * force_field.potential_file is set; callable directly to load another file.  A file named
 * *.alloy or *.setfl (or force_field.potential_format "setfl") is read as a single-element setfl
 * file instead (tables on the file grids, r*phi given directly; the reference reads funcfl only). */
RBMD_API rbmd_status rbmd_force_load_funcfl(rbmd_force* f, const char* path);

/* Water topology for CVFF: n_mol (H,O,H) angle triples, 0-based caller atom ids, the
 * "Angles" section order (rbmd/framework/InitCondition/ModelFileInitCondition.cpp:519-540),
 * plus harmonic bond (k, r0) and angle (k, theta0 in degrees) coefficients of type 0. */
RBMD_API rbmd_status rbmd_force_set_water(rbmd_force* f, int64_t n_mol, const int32_t* hoh_triples_host,
                                 double bond_k, double bond_r0, double angle_k,
                                 double angle_theta0_deg);

/* General CVFF topology (host arrays, 0-based caller atom ids, data-file section order):
 * bonds [n_bonds][2] + type, angles [n_angles][3] + type, dihedrals [n_dihedrals][4] + type, per
 * type coefficients bond (k, r0), angle (k, theta0 in degrees), dihedral (K, sign d = +-1,
 * multiplicity n) of "Bond/Angle/Dihedral Coeffs # harmonic", and the molecule id of every atom.
 * Forces added after the near pass, as ExecutionNVT::ComputeAllForce does for "CVFF"
 * (rbmd/framework/run/ExecutionNVT.cpp:199-215):
 *  - intramolecular Coulomb correction -332.06371 q_i q_j r/r^3 over the other members of
 *    molecules of >= 3 atoms (ComputeSpecialCoulWorklet, RunWorklet.cpp:1386-1437);
 *  - harmonic bonds and angles with per-type coefficients (ExecutionNVT.cpp:467-610);
 *  - with hyper_parameters.extend.special_bonds [w12, w13, w14] in the configuration
 *    (rbmd/framework/application/MDApplication.cpp:157-163): special-bond lists built as
 *    ModelFileInitCondition::SetSpecialBonds does (ModelFileInitCondition.cpp:850-910), LJ pairs
 *    weighted by w instead of excluded within the molecule (RunWorklet.cpp:570-632,816-933), the
 *    Coulomb correction times 1 - w (ComputeSpecialCoulGeneralWorklet, RunWorklet.cpp:1439-1511)
 *    and harmonic dihedrals E = K [1 + d cos(n phi)] (ExecutionNVT.cpp:612-680); without
 *    special_bonds the dihedrals are ignored, as in the reference.
 * Supersedes the water extras of rbmd_force_set_water (SHAKE still uses its triples).  Bonded
 * forces are summed per atom in a fixed order (no atomics).  Callable before or after bind;
 * RBMD_ERR_STATE unless force_field.type is "CVFF". */
typedef struct {
  int64_t n_atoms;
  const int32_t* molecule;                 /* [n_atoms]                                 */
  int64_t n_bonds;
  const int32_t* bonds;                    /* [n_bonds][2]                              */
  const int32_t* bond_type;                /* [n_bonds]                                 */
  int32_t n_bond_types;
  const double* bond_coeffs;               /* [n_bond_types][2] k, r0                   */
  int64_t n_angles;
  const int32_t* angles;                   /* [n_angles][3] i, j (vertex), k            */
  const int32_t* angle_type;
  int32_t n_angle_types;
  const double* angle_coeffs;              /* [n_angle_types][2] k, theta0 (degrees)     */
  int64_t n_dihedrals;
  const int32_t* dihedrals;                /* [n_dihedrals][4]                          */
  const int32_t* dihedral_type;
  int32_t n_dihedral_types;
  const double* dihedral_coeffs;           /* [n_dihedral_types][3] K, sign, multiplicity */
} rbmd_topology;
RBMD_API rbmd_status rbmd_force_set_topology(rbmd_force* f, const rbmd_topology* topology);

/* Attach device atom arrays; sizes the cell grid, neighbour lists and k-space buffers.
 * Replaces ExecutionMD::Init (rbmd/framework/run/ExecutionMD.cpp:117-134). */
RBMD_API rbmd_status rbmd_force_bind(rbmd_force* f, const rbmd_atoms_dev* atoms);

/* Inject the RBE k-samples (integer m vectors, k = 2*pi*m/L) for every replica:
 * m_xyz_host holds n_replicas*P*3 int32.  After this call compute/step use these samples
 * instead of the on-device sampler until rbmd_force_set_ksamples(f, NULL, 0) re-enables it.
 * Replaces the output of RBEPSAMPLE::Fetch_P_Sample (rbmd/framework/model/RBEPSample.h:144-173). */
RBMD_API rbmd_status rbmd_force_set_ksamples(rbmd_force* f, const int32_t* m_xyz_host, int32_t P);

/* Per-sample importance weights (n_replicas*P doubles, host) multiplying each sample's force
 * and energy term; NULL restores unit weights.  Used when the k-samples come from a proposal
 * other than RBE's Gaussian: w = p_gauss(k) / q(k) keeps the estimator unbiased.  No reference
 * counterpart (the reference samples only from the Gaussian, RBEPSample.h:63-175). */
RBMD_API rbmd_status rbmd_force_set_kweights(rbmd_force* f, const double* w_host);

/* Read the k-samples of the last compute (n_replicas*P*3 int32 into host memory).  After
 * rbmd_force_step with the library's own sampler these are the samples drawn for the next step:
 * each step's k-space chain draws the following step's set once its own forces are done. */
RBMD_API rbmd_status rbmd_force_get_ksamples(rbmd_force* f, int32_t* m_xyz_host, int32_t P);

/* Draw the k-samples for `step` with the on-device Metropolis-Hastings sampler (seeded
 * counter RNG; algorithm of RBEPSAMPLE::Fetch_P_Sample/MH_Algorithm) and copy them out. */
RBMD_API rbmd_status rbmd_force_sample_k(rbmd_force* f, int64_t step, int32_t* m_xyz_host, int32_t P);

/* One force evaluation on the caller's stream: cell sort, neighbour list, near force, RBE
 * (or EAM / CVFF extras), sum into atoms->force.  = Force::Execute / ComputeForce
 * (rbmd/framework/run/ExecutionNVT.cpp:179-222). */
RBMD_API rbmd_status rbmd_force_compute(rbmd_force* f, void* stream);

/* Time every choice of the neighbour-list build (0: the shared-memory staged kernel, 1: one warp
 * per atom, or 64, 128, 256 threads per block of the per-atom kernel) and of the force pass (64,
 * 128, 256 threads per block with one thread per atom, or 4 / 8 / 16 / 32 lanes per atom) on the
 * bound system, keep the fastest, and leave the forces of that choice in atoms->force.
 * force_block returns the threads per block, or -G for G lanes per atom.  Config "autotune":
 * true runs it at the first compute; "tuning.list_block" / "tuning.force_block" /
 * "tuning.force_lanes" fix the choices instead (default 0 / 128 / 1).  Lists are identical entry
 * for entry whatever the choice; forces agree to rounding (lanes per atom change the summation
 * order).  No reference counterpart. */
RBMD_API rbmd_status rbmd_force_autotune(rbmd_force* f, void* stream, int32_t* list_block,
                                         int32_t* force_block);

/* Same as rbmd_force_compute with HOST positions in and HOST forces out (n_atoms*3 doubles
 * each); copies are issued on `stream` and the call returns after the force copy landed.
 * This is the call a host-side MD driver (the reference's ExecutionNVT) makes per step. */
RBMD_API rbmd_status rbmd_force_compute_host(rbmd_force* f, const double* pos_host, double* force_host,
                                    void* stream);

/* The same with FP32 host arrays [n_atoms][3], the layout of the reference's
 * vtkm::cont::ArrayHandle<Vec3f> positions and forces (Real = float, rbmd/framework/Types.h:48),
 * so a host driver passes its arrays without converting them: half the PCIe bytes of the FP64
 * call.  Positions are widened to the FP64 master positions on the device and forces narrowed
 * there; the bound device arrays hold the FP64 values afterwards. */
RBMD_API rbmd_status rbmd_force_compute_host_f32(rbmd_force* f, const float* pos_host, float* force_host,
                                                 void* stream);

/* Advance n_steps velocity-Verlet steps in the order of ExecutionNVT::Solve
 * (rbmd/framework/run/ExecutionNVT.cpp:133-159): kick, drift+wrap, SHAKE, force, kick,
 * RATTLE, temperature, thermostat.  Requires vel and mass in the bound atoms. */
RBMD_API rbmd_status rbmd_force_step(rbmd_force* f, int32_t n_steps, void* stream);

/* The thermostat rescale of the last step is applied lazily at the start of the next step;
 * call this to make the bound velocity array current before reading it. */
RBMD_API rbmd_status rbmd_force_sync_velocities(rbmd_force* f, void* stream);

/* Energies of the last compute/step (synchronises the stream). */
RBMD_API rbmd_status rbmd_force_energy(rbmd_force* f, rbmd_energy* out, void* stream);

/* Device status word (RBMD_FLAG_*), synchronises the stream; clear!=0 resets it. */
RBMD_API rbmd_status rbmd_force_status(rbmd_force* f, uint32_t* flags, int32_t clear, void* stream);

/* Full neighbour list of the last compute in caller atom ids: counts[n_atoms] and
 * ids[n_atoms*cap] (row i holds atom i's neighbours), host memory. Returns RBMD_ERR_ARG when
 * cap is smaller than the longest row (counts are still written). Mirrors the id_verletlist /
 * num_verletlist output of ComputeNeighboursWorklet (rbmd/framework/run/worklet/RunWorklet.cpp:40-96). */
RBMD_API rbmd_status rbmd_force_get_neighbors(rbmd_force* f, int32_t* counts_host, int32_t* ids_host,
                                     int64_t cap);

/* RBL lists of the last compute (neighbor.type "RBL"): per caller atom the number of core pairs
 * (d < r_core) and of kept shell pairs (every pice-th pair in r_core <= d < cut_off, in the
 * reference's traversal order); rbmd_force_get_neighbors returns the pairs themselves, core first.
 * sizes[5] = rs_num, rc_num, pice_num of the reference's sizing formulas for replica 0, then the
 * library's core and shell capacities.  Mirrors num_verletlist[2] of
 * ComputeRBLNeighboursOnceWorklet (rbmd/framework/run/worklet/RunWorklet.cpp:634-708) and the
 * sizes of ExecutionMD::ComputeRBLNearForce (rbmd/framework/run/ExecutionMD.cpp:460-486). */
RBMD_API rbmd_status rbmd_force_get_rbl(rbmd_force* f, int32_t* ncore_host, int32_t* nshell_host,
                                        int64_t* sizes);

/* Structure factors of the last compute: rho[n_replicas*P*2] (Re, Im) doubles, host memory,
 * with the phase origin at each box's lo corner (|rho| equals the reference's
 * ComputePnumberChargeStructureFactorWorklet + ReduceByKey result,
 * rbmd/framework/run/worklet/RunWorklet.cpp:1616-1677). */
RBMD_API rbmd_status rbmd_force_get_rhok(rbmd_force* f, double* rho_host, int32_t P);

/* Per-phase device timing with CUDA events recorded on the stream each phase runs on
 * (0 integrate, 1 cell sort, 2 structure factors, 3 neighbour list, 4 near/EAM force pass,
 * 5 constraints and intramolecular terms, 6 k sampler, 7 RBE force).  enable resets the accumulators; phase_ms returns the summed
 * milliseconds and the number of timed intervals per phase since then.  No reference
 * counterpart beyond its vtkm::cont::Timer aliases (rbmd/framework/Timer.h:32). */
RBMD_API rbmd_status rbmd_force_profile(rbmd_force* f, int32_t enable);
RBMD_API rbmd_status rbmd_force_phase_ms(rbmd_force* f, double* ms, int64_t* counts, int32_t n);

/* Number of neighbour-list builds since bind, counted per replica (with a Verlet skin a
 * replica's list is rebuilt only when one of its atoms moved more than skin/2, and the other
 * replicas keep theirs; the reference rebuilds on every force call). */
RBMD_API rbmd_status rbmd_force_list_builds(rbmd_force* f, int64_t* builds);

/* Library/kernel description for diagnostics: number of kernels the last compute or step
 * launched per step. */
RBMD_API rbmd_status rbmd_force_launch_count(rbmd_force* f, int32_t* kernels_per_step);

RBMD_API void rbmd_force_destroy(rbmd_force* f);

/* Structure factors rho_k = sum_j q_j exp(i 2 pi m_k . (r_j - lo) / L) of n atoms in one box
 * (device positions [n*3] and charges [n]) for P integer vectors m (device int32 [P*3]) into
 * rho (device double [P*2], Re then Im), enqueued on `stream`, with no device allocation: the
 * scratch lives in a static device array of the library (8 MiB per device, kept until exit).
 * For callers that cannot allocate device memory at that point: an engine that owns all device
 * memory through its own pool or a fixed budget, or a step loop that cannot take the device-wide
 * synchronisation of cudaFree.  Limits: n <= 262144, P <= 1024, else
 * RBMD_ERR_ARG.  All calls on a device share the array: calls that overlap on the GPU race.
 * Every call made outside stream capture resolves the array's address in the current context
 * (so a device reset leaves nothing stale); the first call on each device, and the first after
 * a reset, should precede any stream capture, since a call during capture only reuses the
 * address recorded for its context (RBMD_ERR_CUDA if there is none).  A CUDA error already
 * pending from the caller's earlier work is returned as RBMD_ERR_CUDA before anything is
 * launched.  NaN positions give unspecified rho.  No counterpart in the reference. */
RBMD_API rbmd_status rbmd_rhok_noalloc(const double* pos_dev, const double* charge_dev, int32_t n,
                                       const rbmd_box* box, const int32_t* m_dev, int32_t P,
                                       double* rho_dev, void* stream);

/* The learned k-proposal network (16 -> 64 -> 64 -> 1, tanh, BF16 operands on the tensor
 * cores, FP32 accumulation) on `groups` groups of 256 rows, all pointers on the device:
 * params[5313] (W1[64][16], b1[64], W2[64][64], b2[64], w3[64], b3), x[groups*256][16] inputs,
 * h[groups*256] outputs.  With train != 0 also the group losses
 * loss[g] = log sum_b wbin_b e^{h_b} + log sum_b cbin_b e^{-h_b} and the gradient of their mean
 * into grad[5313].  status receives 0x80 when an internal wait gave up.  train < 0 evaluates h
 * alone on the CUDA cores instead, as the sampler does every step (same BF16 roundings, FP32 sums
 * in another order; no shared memory, so it shares SMs with a running near pass).  Synchronises
 * the stream.
 * No reference counterpart (the reference samples k from the Gaussian only,
 * rbmd/framework/model/RBEPSample.h:63-175). */
RBMD_API rbmd_status rbmd_proposal_mlp_eval(const float* params, const float* x, const float* wbin,
                                            const float* cbin, int32_t groups, int32_t train, float* h,
                                            double* loss, float* grad, uint32_t* status, void* stream);

/* Options and outcome of rbmd_force_train_proposal. */
typedef struct {
  int32_t n_snapshots;     /* snapshots of the bound system (groups of the training batch)       */
  int32_t steps_between;   /* MD steps (rbmd_force_step) before each snapshot; 0: static system  */
  int32_t k_per_snapshot;  /* k-vectors drawn from the Gaussian per snapshot                      */
  int32_t iterations;      /* Adam steps on the full batch                                       */
  float learning_rate;
  uint64_t seed;           /* network initialisation and k draws                                 */
} rbmd_train_opts;

typedef struct {
  double loss_gauss;       /* mean group loss of h = 0 (the Gaussian proposal)                    */
  double loss_first;       /* after the first Adam step                                          */
  double loss_final;       /* after the last Adam step                                           */
  double loss_optimum;     /* lower bound: h_b = log sqrt(C_b / W_b) per snapshot                 */
  double variance_ratio;   /* exp(loss_final - loss_gauss): learned / Gaussian force variance     */
  double seconds;          /* wall time of data generation + training                            */
} rbmd_train_report;

/* Train the learned k-proposal (coulomb.proposal "learned") on the bound system: for each of
 * n_snapshots snapshots (advancing the system by steps_between MD steps first), draw
 * k_per_snapshot vectors from RBE's Gaussian, compute their exact structure factors rho_k (the
 * full Ewald sum's terms) and the squared norm of each sample's force field, bin them into the
 * per-|k| variance weights C_b and the snapshot's spectrum; then fit the network by Adam on the
 * log force variance of the reweighted proposal, all on the GPU (tcgen05 forward/backward).
 * Replica 0 provides the data.  Afterwards every compute/step draws its k-samples from the
 * trained proposal with importance weights p/q.  No reference counterpart. */
RBMD_API rbmd_status rbmd_force_train_proposal(rbmd_force* f, const rbmd_train_opts* opts,
                                               rbmd_train_report* report, void* stream);

/* Read (get_host != NULL) and/or replace (set_host != NULL) the 5313 network parameters of the
 * learned proposal; setting parameters marks the proposal as trained.  No reference counterpart. */
RBMD_API rbmd_status rbmd_force_proposal_params(rbmd_force* f, float* get_host, const float* set_host);

/* k-space (RBE) force of the last compute per caller atom, far_host[n_atoms*3] (zero for
 * uncharged atoms; qqr2e applied).  Two evaluations with different k-sets give the estimator's
 * noise.  Mirrors the far force of ExecutionNVT::EleNewForce (rbmd/framework/run/ExecutionNVT.cpp:717-733). */
RBMD_API rbmd_status rbmd_force_get_far(rbmd_force* f, double* far_host);

/* ---- LAMMPS data files (the reference's read_data input) ------------------------------------
 * rbmd_data_read parses a data file as ModelFileInitCondition does
 * (rbmd/framework/InitCondition/ModelFileInitCondition.cpp:120-605): header counts, Masses,
 * Pair Coeffs, Bond/Angle/Dihedral Coeffs, Atoms in style "atomic" | "charge" | "full", Bonds,
 * Angles, Dihedrals, Velocities; ids, types and molecules 0-based, atoms ordered by id; unit "LJ" sets every mass
 * to 1 as the reference does.  The accessors copy into caller-allocated host arrays (NULL skips
 * an array): positions/velocities [n][3], charge/mass [n], type/molecule [n], image flags [n][3]
 * (optional columns after the coordinates, 0 when absent), per-type masses / epsilon / sigma
 * [n_atom_types], bonds [n_bonds][2], angles [n_angles][3] (caller atom ids), bond / angle
 * coefficients [types][2] = (k, r0 | theta0 in degrees).  rbmd_data_write writes the same format
 * (checkpoints that double as inputs; image flags kept). */
typedef struct rbmd_data rbmd_data;
typedef struct {
  int64_t n_atoms, n_bonds, n_angles;
  int32_t n_atom_types, n_bond_types, n_angle_types;
  int32_t has_velocities, has_pair_coeffs, has_masses;
  rbmd_box box;
  int64_t n_dihedrals;
  int32_t n_dihedral_types;
} rbmd_data_info;
RBMD_API rbmd_status rbmd_data_read(const char* path, const char* atom_style, const char* unit, rbmd_data** out,
                                    rbmd_data_info* info);
RBMD_API rbmd_status rbmd_data_atoms(const rbmd_data* d, double* pos, double* vel, double* charge, int32_t* type,
                                     int32_t* molecule, double* mass, int32_t* image);
RBMD_API rbmd_status rbmd_data_types(const rbmd_data* d, double* mass_by_type, double* epsilon, double* sigma);
RBMD_API rbmd_status rbmd_data_topology(const rbmd_data* d, int32_t* bonds, int32_t* bond_type, int32_t* angles,
                                        int32_t* angle_type, double* bond_coeffs, double* angle_coeffs);
/* Dihedrals [n_dihedrals][4] (caller atom ids), their types and the harmonic coefficients
 * [n_dihedral_types][3] = (K, sign, multiplicity) of "Dihedral Coeffs". */
RBMD_API rbmd_status rbmd_data_dihedrals(const rbmd_data* d, int32_t* dihedrals, int32_t* dihedral_type,
                                         double* dihedral_coeffs);
RBMD_API void rbmd_data_free(rbmd_data* d);
RBMD_API rbmd_status rbmd_data_write(const char* path, const char* atom_style, const rbmd_data_info* info,
                                     const double* pos, const double* vel, const double* charge,
                                     const int32_t* type, const int32_t* molecule, const int32_t* image,
                                     const double* mass_by_type, const double* epsilon, const double* sigma,
                                     const int32_t* bonds, const int32_t* angles);

/* Every section the reader returns, including bond / angle / dihedral types and the harmonic
 * coefficients of "Bond/Angle/Dihedral Coeffs" (a checkpoint of a molecular system that reads
 * back identically).  NULL arrays are left out; missing term types are written as type 1.  Counts
 * come from `info` (n_bonds, n_bond_types, ... n_dihedral_types).  rbmd_data_write is this call
 * without types, coefficients and dihedrals. */
typedef struct {
  const double *pos, *vel, *charge;
  const int32_t *type, *molecule, *image;
  const double *mass_by_type, *epsilon, *sigma;
  const int32_t *bonds, *bond_type;
  const double* bond_coeffs;       /* [n_bond_types][2] k, r0 */
  const int32_t *angles, *angle_type;
  const double* angle_coeffs;      /* [n_angle_types][2] k, theta0 (degrees) */
  const int32_t *dihedrals, *dihedral_type;
  const double* dihedral_coeffs;   /* [n_dihedral_types][3] K, sign, multiplicity */
} rbmd_data_arrays;
RBMD_API rbmd_status rbmd_data_write_arrays(const char* path, const char* atom_style, const rbmd_data_info* info,
                                            const rbmd_data_arrays* arrays);

/* Version string of the library build. */
RBMD_API const char* rbmd_version(void);

/* Text of the last host-side error (CUDA call, config key), empty when none. */
RBMD_API const char* rbmd_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* RBMD_FORCE_H */
