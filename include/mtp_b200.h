/*
 * mtp_b200.h - C ABI of the B200 Moment Tensor Potential engine.
 *
 * This library replaces the reference's compiled-XLA bridge
 * (pair_style_files/zero_overhead.{hpp,cpp}: a CPython/NumPy singleton that
 * deserialises a jax.export executable and calls it every MD step) with
 * hand-written sm_100a CUDA kernels behind plain C functions.  No torch,
 * CPython or C++ types cross this boundary: pointers, sizes and int status
 * codes only.  No C++ exception escapes any function.
 *
 * Conventions (identical to the reference evaluator jax_backend.py):
 *   - a neighbour slot of centre atom i holds r_ij = x_j - x_i, the owner
 *     index j of the neighbour, and its species t_j; a slot contributes
 *     when t_j >= 0 and |r_ij| < max_dist of the potential
 *     (jax_backend.py:83-90);
 *   - slots whose owner index j is outside [0, natoms) still contribute to
 *     E_i but their reaction force is dropped (jax_backend.py:292-299);
 *   - forces F_k = sum_s dE_k/dr_ks - sum_{(i,s): j_is = k} dE_i/dr_is
 *     (jax_backend.py:263-303);
 *   - species are 0-based (LAMMPS type - 1, pair_jax_mtp.cpp:97).
 *
 * Virial conventions:
 *   - mtp_compute*: LAMMPS virial in energy units, W = -sum r (x) dE/dr,
 *     symmetrised, order xx, yy, zz, xy, xz, yz (what Pair::virial holds);
 *   - mtp_execute_potential: the reference's `stress` output unchanged,
 *     sym(sum r (x) dE/dr) / V in order xx, yy, zz, yz, xz, xy
 *     (jax_backend.py:355-360, consumed at pair_jax_mtp.cpp:203-205).
 *
 * Thread safety: a handle is used by one host thread at a time.  Each handle
 * owns its device buffers and one CUDA stream (settable).
 */
#ifndef MTP_B200_H
#define MTP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MTP_B200_ABI_VERSION 1

/* Status codes returned by every entry point. */
typedef enum mtp_status {
  MTP_OK = 0,
  MTP_E_INVALID = 1,    /* bad argument (null pointer, negative size, ...)          */
  MTP_E_FORMAT = 2,     /* malformed .mtp file or unsupported table structure       */
  MTP_E_CAPACITY = 3,   /* natoms > max_atoms or a row longer than max_nbr          */
  MTP_E_SPECIES = 4,    /* a species index outside [0, species_count)               */
  MTP_E_NONFINITE = 5,  /* NaN/Inf produced on the device                           */
  MTP_E_CUDA = 6,       /* CUDA runtime error (text in mtp_last_error)              */
  MTP_E_NODEVICE = 7,   /* no usable CUDA device                                    */
  MTP_E_OOM = 8         /* device allocation failed                                 */
} mtp_status;

/* Arithmetic of the evaluator. */
typedef enum mtp_precision {
  MTP_PRECISION_FP64 = 0,   /* everything in FP64 (the drop-in)                       */
  MTP_PRECISION_MIXED = 1   /* FP32 radial/moments/contractions; FP64 energy, virial,
                               force accumulation                                      */
} mtp_precision;

/* Output selection flags for mtp_compute*. */
#define MTP_EFLAG 1   /* total energy           */
#define MTP_VFLAG 2   /* global virial          */
#define MTP_EATOM 4   /* per-atom energies      */
#define MTP_VATOM 8   /* per-atom virial        */
#define MTP_REUSE_NEIGHBORS 16  /* mtp_compute_device: the neighbour indices are those of the
                                   previous call; skip rebuilding the incoming-slot lists  */

typedef struct mtp_handle mtp_handle;

/* Library ABI version (MTP_B200_ABI_VERSION of the build). */
int mtp_abi_version(void);

/*
 * Create an evaluator from an .mtp potential file.
 * Replaces PairJaxMTP::settings + init_style + ZeroOverheadContext
 * (pair_jax_mtp.cpp:228-245, 264-282; zero_overhead.cpp:159-169, 317-320):
 * max_atoms and max_nbr are the pair style's MAX_ATOMS and
 * MAX_ATOMS_PER_NEIGHBOR capacities, cutoff its MTP_CUTOFF, debug_level its
 * DEBUG_LEVEL (0 silent, 1 summary at destroy, 2 per-call timing to stderr).
 * The reference takes a .bin export here; a path ending in ".bin" is
 * rejected with MTP_E_FORMAT.
 */
int mtp_create(const char* mtp_path, int max_atoms, int max_nbr, double cutoff, int debug_level,
               int precision, mtp_handle** out);

/* Release every device buffer of the handle. */
void mtp_destroy(mtp_handle* h);

/* Text of the last error on this handle (or of the last failed mtp_create when h is NULL). */
const char* mtp_last_error(const mtp_handle* h);

/* Use this CUDA stream (a cudaStream_t) for all work of the handle; NULL is the
 * legacy default stream (as in the CUDA runtime).  A new handle works on a
 * non-blocking stream of its own; mtp_use_own_stream returns to it. */
int mtp_set_stream(mtp_handle* h, void* cuda_stream);
int mtp_use_own_stream(mtp_handle* h);

/* Basis sizes of the loaded potential: out[0..7] = species_count, radial_funcs_count,
 * radial_basis_size, alpha_moments_count, alpha_index_basic_count,
 * alpha_index_times_count, alpha_scalar_moments, max monomial degree. */
int mtp_get_info(const mtp_handle* h, int* out8);

/* Call statistics: out4 = {host-buffer calls (mtp_compute and the bridge),
 * their total host time in ms, CUDA graphs captured for mtp_compute, graph
 * replays}.  Below 65,536 atoms, mtp_compute with page-locked host buffers
 * (mtp_host_alloc, cudaHostRegister) captures its copies and kernels as one
 * CUDA graph on the second consecutive call with the same arguments and
 * replays it while they repeat. */
int mtp_get_stats(const mtp_handle* h, double* out4);

/* Replace the coefficients (training updates): species [S], moment [Sa], radial [S*S*R*K]
 * in .mtp order.  Any pointer may be NULL to keep the current values. */
int mtp_set_coeffs(mtp_handle* h, const double* species_coeffs, const double* moment_coeffs,
                   const double* radial_coeffs);

/*
 * Drop-in for ZeroOverheadManager::execute_potential (zero_overhead.hpp:58-64,
 * zero_overhead.cpp:171-272), same arguments and meaning: per-atom row
 * pointers of r_ij (3 doubles per neighbour), neighbour owner indices and
 * neighbour species, neighbour counts, cell volume.  Outputs the total energy,
 * forces[i][0..2] for i < natoms, and stress[6] in the reference's convention
 * (see above).  Returns MTP_OK (the reference returned bool true) or an error.
 */
int mtp_execute_potential(mtp_handle* h, int natoms, int nneigh_total,
                          const double* const* atom_positions, const int* atom_types,
                          const int* const* neighbor_lists, const int* neighbor_counts,
                          const int* const* neighbor_types_lists, double volume,
                          double* energy, double** forces, double* stress);

/*
 * Flat host-buffer evaluation (the pair style's fast path).
 * itypes [natoms]; rijs [natoms][nbr_stride][3]; js, jtypes [natoms][nbr_stride];
 * counts [natoms] (NULL: every slot of a row is examined, empty slots have
 * jtype < 0).  nbr_stride <= max_nbr.  Outputs selected by flags; pointers of
 * unselected outputs may be NULL.  forces [natoms][3] is always written.
 * virial [6] (LAMMPS order), eatom [natoms], vatom [natoms][6].
 * Synchronous: returns when results are in host memory.  From 65,536 atoms on,
 * the inputs are copied in atom chunks on a second, library-owned stream while
 * the evaluation runs on the chunks already copied (pinned host buffers let
 * the copies overlap; results are bitwise those of mtp_compute_device).  Below
 * that, with every host buffer page-locked and the handle on a non-default
 * stream, the second consecutive call with the same arguments is captured as
 * one CUDA graph (copies, kernels, read-backs) and replayed while the
 * arguments repeat; the buffers' contents may change between calls.
 */
int mtp_compute(mtp_handle* h, int natoms, int nbr_stride, const int* itypes, const double* rijs,
                const int* js, const int* jtypes, const int* counts, int flags, double* energy,
                double* forces, double* virial, double* eatom, double* vatom);

/*
 * Host-buffer evaluation from positions: the neighbour rows are built on the
 * device, so a pair style sends positions and its neighbour list instead of
 * packed r_ij rows (the host loop of PairJaxMTP::compute,
 * pair_jax_mtp.cpp:110-167, moves to the GPU).
 *   x [nall][3]        positions of the nlocal local atoms, then the ghosts
 *   species [nall]     0-based species of every atom
 *   owner [nall]       local index of each atom's owner: i for i < nlocal, the
 *                      local atom with the ghost's tag, or -1 (the ghost then
 *                      has species -1 in the rows and contributes nothing,
 *                      pair_jax_mtp.cpp:137-151)
 *   neigh [nlocal][list_stride]  candidate neighbour indices into [0, nall)
 *                      (the full list, skin included); numneigh [nlocal]
 * Candidates closer than the handle's cutoff are kept in list order with
 * r_ij = x_j - x_i, exactly as a host loop packs them, so the results are
 * bitwise those of mtp_compute on the rows that loop would build.  More than
 * max_nbr kept candidates in a row: MTP_E_CAPACITY.  Outputs as mtp_compute;
 * synchronous.  With every buffer page-locked and the handle on a non-default
 * stream, the second consecutive call with the same arguments is captured as
 * one CUDA graph and replayed while they repeat, as for mtp_compute.
 */
int mtp_compute_positions(mtp_handle* h, int nlocal, int nall, const double* x, const int* species,
                          const int* owner, int list_stride, const int* neigh, const int* numneigh,
                          int flags, double* energy, double* forces, double* virial, double* eatom,
                          double* vatom);

/*
 * Device-pointer variant of mtp_compute_positions: the same arguments in
 * device memory, outputs as mtp_compute_device (energy [1], forces
 * [nlocal][3], virial [6], optional eatom/vatom), enqueued on the handle's
 * stream without synchronising; device-side errors (an overfull row sets
 * MTP_E_CAPACITY) are read with mtp_sync_status.  This is the call of a
 * pair style whose positions, species and neighbour list already live on
 * the GPU (the reference's README.md:48 plans a Kokkos pair style; LAMMPS's
 * KOKKOS package keeps x, type and the neighbour list in device views).
 */
int mtp_compute_positions_device(mtp_handle* h, int nlocal, int nall, const double* d_x,
                                 const int* d_species, const int* d_owner, int list_stride,
                                 const int* d_neigh, const int* d_numneigh, int flags,
                                 double* d_energy, double* d_forces, double* d_virial,
                                 double* d_eatom, double* d_vatom);

/*
 * Device-pointer variant of mtp_compute for PyTorch and CUDA-graph capture:
 * every pointer is device memory; work is enqueued on the handle's stream and
 * the call returns without synchronising.  energy [1], virial [6].
 * Device-side error flags are read with mtp_sync_status.
 */
int mtp_compute_device(mtp_handle* h, int natoms, int nbr_stride, const int* d_itypes,
                       const double* d_rijs, const int* d_js, const int* d_jtypes,
                       const int* d_counts, int flags, double* d_energy, double* d_forces,
                       double* d_virial, double* d_eatom, double* d_vatom);

/* Synchronise the handle's stream and report device-side error flags
 * (MTP_E_NONFINITE, MTP_E_SPECIES) raised since the last call. */
int mtp_sync_status(mtp_handle* h);

/*
 * Batched evaluation of many configurations in one launch (training
 * forward).  Atoms of all configurations are concatenated; js holds global
 * atom indices; cfg_of_atom [natoms] maps atoms to configurations
 * [0, nconfig).  Outputs (device): energy [nconfig], forces [natoms][3],
 * stress [nconfig][6] in the reference's convention (sym(sum r g)/V, order
 * xx,yy,zz,yz,xz,xy) using volumes [nconfig] (device), as the reference
 * training code computes it (motep_original_files/jax_engine/jax.py:76-91).
 */
int mtp_compute_batch_device(mtp_handle* h, int natoms, int nbr_stride, int nconfig,
                             const int* d_itypes, const double* d_rijs, const int* d_js,
                             const int* d_jtypes, const int* d_counts, const int* d_cfg_of_atom,
                             const double* d_volumes, double* d_energy, double* d_forces,
                             double* d_stress);

/*
 * Adjoint of mtp_compute_batch_device with respect to the coefficients
 * (the gradient jax.grad takes of the training loss,
 * training/motep_jax_train_function.py:67-87, 191).  Given upstream
 * gradients gE [nconfig], gF [natoms][3], gS [nconfig][6] (device) for the
 * same inputs, writes (device) dL/d species_coeffs [S], dL/d moment_coeffs
 * [Sa] and dL/d radial_coeffs [S*S*R*K].  Second derivatives of the forces
 * and stress are included.  Deterministic.
 */
int mtp_adjoint_batch_device(mtp_handle* h, int natoms, int nbr_stride, int nconfig,
                             const int* d_itypes, const double* d_rijs, const int* d_js,
                             const int* d_jtypes, const int* d_counts, const int* d_cfg_of_atom,
                             const double* d_volumes, const double* d_gE, const double* d_gF,
                             const double* d_gS, double* d_gspecies, double* d_gmoment,
                             double* d_gradial);

/* Launch shape of the evaluation kernel: threads per block (128/256/512),
 * blocks per SM (0 = as many as fit) and atoms evaluated together per block
 * (0 = chosen by occupancy, or 1/2/4; FP64 supports 1/2).  Used by the
 * autotuner. */
int mtp_set_launch(mtp_handle* h, int threads_per_block, int blocks_per_sm, int atoms_per_block);

/* Last evaluation kernel's launch: out5 = threads, blocks, dynamic shared bytes,
 * blocks per SM, atoms per block. */
int mtp_get_launch(const mtp_handle* h, int* out5);

/*
 * Parse an .mtp file on the host only (no device needed) and report its
 * basis sizes in the layout of mtp_get_info.  Used to validate files.
 */
int mtp_parse_info(const char* mtp_path, int* out8, char* err, int err_len);

/*
 * Host execution of the contraction schedule for one atom (no device needed;
 * a test hook for the table preprocessing).  basic [alpha_index_basic_count]
 * moments in, moments [alpha_moments_count] and dE/dmoment [alpha_moments_count]
 * out, using the handle-free preprocessing of the file and the schedule for
 * threads_per_block lanes whose entry order is tuned for access_width-byte
 * operand loads (4, 8 or 16).
 */
int mtp_schedule_emulate(const char* mtp_path, int threads_per_block, int access_width, const double* basic,
                         double* moments, double* dmoments, double* energy_part);

/*
 * Device neighbour rows with a cell list (positions d_pos [natoms][3] on the
 * device, cell9 = the three lattice vectors as rows, host).  For every atom,
 * the slots hold every periodic image within `cutoff`: owner index (d_js),
 * image code (d_image, for mtp_pack_rij_device), species (d_jtypes), and the
 * count (d_counts); unused slots get index -1 and species -1.  Rows longer
 * than nbr_stride are truncated and reported as MTP_E_CAPACITY by
 * mtp_sync_status (the reference drops such neighbours silently,
 * pair_jax_mtp.cpp:132).  Each cell edge must be at least `cutoff` long.
 * Replaces the host packing of pair_jax_mtp.cpp:110-167 for device-resident MD.
 */
int mtp_neighbors_device(mtp_handle* h, int natoms, const double* d_pos, const double* cell9,
                         const int* d_types, double cutoff, int nbr_stride, int* d_js, int* d_image,
                         int* d_jtypes, int* d_counts);

/* r_ij = x_j - x_i + image . cell for the rows of mtp_neighbors_device (device). */
int mtp_pack_rij_device(mtp_handle* h, int natoms, int nbr_stride, const double* d_pos, const double* cell9,
                        const int* d_js, const int* d_image, const int* d_counts, double* d_rijs);

/* Velocity Verlet in LAMMPS 'metal' units (A, ps, eV, amu): stage 1 = half kick
 * + drift, stage 2 = half kick.  masses [species] in amu (host). */
int mtp_verlet_device(mtp_handle* h, int natoms, double* d_x, double* d_v, const double* d_f, const int* d_types,
                      const double* masses, int nmasses, double dt, int stage);

/* Time the evaluation kernel with CUDA events on the handle's stream:
 * enable = 1 starts accumulating, mtp_profile_read returns the total kernel
 * milliseconds and launch count since enabling (synchronises). */
int mtp_profile(mtp_handle* h, int enable);
int mtp_profile_read(mtp_handle* h, double* eval_ms, int* eval_launches);

/*
 * No counterpart in the reference.
 *
 * Allocation-free evaluation for callers that cannot let a library allocate
 * device memory: code running while a stream is captured into a CUDA graph
 * (cudaMalloc is illegal during capture), code that must not synchronise the
 * device (cudaMalloc and cudaFree can), and hosts whose memory pool owns the
 * whole GPU.  Same inputs and meaning as mtp_compute_device, outputs energy [1],
 * forces [natoms][3] and the LAMMPS virial [6] (device pointers).  It calls no
 * cudaMalloc, cudaFree or allocating library routine: its scratch is one
 * fixed array of about 8.5 MB in the library's device memory, held by every
 * GPU that loads the library until the process exits, and it uses only the
 * contraction schedules the handle already uploaded.  Limits: at most
 * MTP_NOALLOC_MAX_ATOMS atoms and MTP_NOALLOC_MAX_SLOTS neighbour slots
 * (natoms * nbr_stride); larger inputs, or a basis whose value space does
 * not fit in shared memory, return MTP_E_CAPACITY.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress), so make
 * that first call before any stream capture.  The address is kept for the
 * life of the process: after cudaDeviceReset (or anything else that destroys
 * the device's primary context) it is stale, so do not use this entry point
 * again in that process.  All calls share the array:
 * calls that overlap on the GPU (several streams, several handles) race.
 */
#define MTP_NOALLOC_MAX_ATOMS 16384
#define MTP_NOALLOC_MAX_SLOTS 262144
int mtp_compute_device_noalloc(mtp_handle* h, int natoms, int nbr_stride, const int* d_itypes,
                               const double* d_rijs, const int* d_js, const int* d_jtypes,
                               const int* d_counts, double* d_energy, double* d_forces,
                               double* d_virial);

/* Peak FP64 / FP32 FMA throughput of device 0 measured by an FMA-chain kernel
 * (TFLOP/s, an FMA counted as 2 flops).  Used for the roofline. */
int mtp_measure_fma_peak(double* fp64_tflops, double* fp32_tflops);

/*
 * Page-locked host memory for the host-buffer entry points.  A caller that
 * packs its rows (rijs, js, jtypes, counts, itypes) and receives its outputs
 * in these buffers lets mtp_compute move them by DMA instead of through the
 * driver's staging copy of pageable memory.  The reference's pool refilled
 * pageable NumPy arrays every step (zero_overhead.cpp:61-117); this replaces
 * that pool's storage.  bytes == 0 gives *out == NULL.  Errors: MTP_E_INVALID,
 * MTP_E_OOM, MTP_E_CUDA (text in mtp_last_error(NULL)).  mtp_host_free(NULL)
 * is a no-op.
 */
int mtp_host_alloc(size_t bytes, void** out);
int mtp_host_free(void* p);

#ifdef __cplusplus
}
#endif

#endif /* MTP_B200_H */
