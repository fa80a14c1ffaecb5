/*
 * melon3d_gpu.h — extensions of the GPU world beyond Melon3D's C API.
 *
 * None of these has a counterpart in the reference's public header; they
 * exist because a GPU world is used differently from a CPU one:
 *  - batch readback of every body slot in one copy (the per-body getters of
 *    melon3d.h stay available and exact, but cost one call per body);
 *  - device-side timing of the last step (CUDA events on the world's stream);
 *  - an error status word (kernels never trap: a failed launch, an exhausted
 *    allocation or a bounded wait that ran out is reported here);
 *  - the snapshot functions of melon3d_debug.h (m3d_dbg_*), which the test
 *    suite uses to compare the world with the reference field by field.
 * All functions take the world created by m3d_world_create (melon3d.h).
 */
#ifndef MELON3D_GPU_H
#define MELON3D_GPU_H

#include "melon3d.h"
#include "melon3d_debug.h"

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define M3D_GPU_OK 0
#define M3D_GPU_ERR_CUDA (-1)    /* a CUDA call failed; see m3d_gpu_last_error_string */
#define M3D_GPU_ERR_ALLOC (-2)   /* device memory could not be grown */
#define M3D_GPU_ERR_HASH (-3)    /* a pair hash table overflowed (internal sizing bug) */
#define M3D_GPU_ERR_LIMIT (-4)   /* input larger than a fixed scratch block allows */
#define M3D_GPU_ERR_PENDING (-5) /* API edits not yet uploaded to the device */
#define M3D_GPU_ERR_ARGUMENT (-6) /* a required pointer was NULL */
#define M3D_GPU_ERR_WAIT (-7)    /* a bounded device-side wait ran out (the step's results are suspect) */

/* Number of body slots (live or free); slot i is body index i. */
M3D_API int32_t m3d_gpu_body_capacity(m3d_world* world);

/* Copy position (xyz) and rotation (xyzw) of the first `capacity` slots,
 * straight from device memory, into caller-owned host arrays
 * (3*capacity and 4*capacity floats).  Either pointer may be NULL. */
M3D_API void m3d_gpu_read_poses(m3d_world* world, float* positions, float* rotations, int32_t capacity);

/* Device time of the last m3d_world_step, milliseconds (CUDA events on the
 * world's stream around the step's work, uploads included). */
M3D_API float m3d_gpu_last_step_device_ms(m3d_world* world);

/* Work counters of the last step, in this order: activeEntries,
 * stableEntries, activeOversized, stableOversized, cellRuns, gridPairs,
 * oversizedPairs, newContacts, removedContacts, removalEndEvents,
 * beginEvents, endEvents, anyAwakeDynamic, islandCount, touchingContacts,
 * awakeIslands, islandContacts, islandJoints, islandBodies, stableDirty,
 * bodyCount, awakeBodyCount, hashFailures, colouredIslands, serialIslands,
 * freeIslands, waitErrors, contactCount, giantIslands, keptStable,
 * keptStableOversized, keptContacts, tinyIslands, warpIslands, islandPoints,
 * serialBodies, serialContacts, sleptBodies (counted only while a tape
 * records).  Returns how many counters exist (writes at most capacity). */
M3D_API int32_t m3d_gpu_step_counters(m3d_world* world, uint32_t* out, int32_t capacity);

/* Coloured islands (>= 300 contacts, solved with the reference's greedy
 * colouring) with at least `contacts` contacts are solved by all SMs in one
 * cooperative launch instead of one CTA each (default 32768; values below 300
 * mean 300).  Results are identical either way; only the speed differs. */
M3D_API void m3d_gpu_set_giant_island_contacts(m3d_world* world, int32_t contacts);

/* Stage profile of the last giant-island solve (profiling aid, no
 * counterpart in the reference): out[0..4] = device ns spent building the
 * incidence lists, colouring, bucketing by colour, levelling the overflow
 * bucket (and preparing joints), and running the substeps; out[5] = colours
 * used, out[6] = contacts in the serial overflow bucket, out[7] = its levels;
 * out[8..14] = device ns of the substep stages summed over the substeps:
 * integration + preparation, coloured normal sweeps, overflow normal sweeps
 * (and joints), friction, reconstruction, coloured velocity sweeps, overflow
 * velocity sweep (and joints).  Returns the count written (at most 15; 0 if
 * the world never solved a giant island). */
M3D_API int32_t m3d_gpu_giant_profile(m3d_world* world, double* out, int32_t capacity);

/* Batch of worlds (no counterpart in the reference).  Packs `count` worlds
 * built with melon3d.h and not stepped yet (same gravity, iterations, cell
 * size and sleep setting) into one new world whose step advances all of them
 * at once.  Each world's result is the one its own step would give: its
 * contacts keep their own order, its stable tier its own schedule, and no
 * pair spans two worlds.  Body i of world k is body slot
 * m3d_gpu_batch_first_body(batch, k) + i of the batch, with the generation it
 * had; getters, setters, poses, profile and m3d_gpu_* work on the batch.
 * Bodies and joints cannot be created or destroyed in a batch and the
 * world queries return no hit; contact events are the narrowphase begin/end
 * events of all worlds together.  The source worlds stay valid and
 * independent.  Limits: 2^24 worlds; cell coordinates within +-2^(b-1) cells
 * where b = floor((63 - ceil(log2 count)) / 3) (17 bits for 4096 worlds).
 * Returns NULL on failure (message on stderr). */
M3D_API m3d_world* m3d_gpu_batch_create(m3d_world* const* worlds, int32_t count);
M3D_API int32_t m3d_gpu_batch_world_count(m3d_world* batch);
/* first body slot of world k; k == count gives the total slot count */
M3D_API int32_t m3d_gpu_batch_first_body(m3d_world* batch, int32_t k);

/* Online autotuning (no counterpart in the reference).  The kernel that
 * solves a serial island - one warp per island, or one thread per island for
 * islands of a few contacts without joints - is chosen by two thresholds;
 * every choice gives the same results bit for bit, so m3d_gpu_autotune tries
 * the candidates on the world's own next steps (each for stepsPerTrial steps,
 * two interleaved rounds), keeps the one with the lowest median device time,
 * and appends it to the file named by M3D_AUTOTUNE_CACHE (one line per GPU
 * model, body-count and world-count magnitude), where a later call with the
 * same key finds it and applies it at once (returns 1; else 0).
 * stepsPerTrial <= 0 restores the defaults.  m3d_gpu_autotune_state returns
 * 0 (not tuning), 1 (trials running) or 2 (a choice applied) and the current
 * thresholds. */
M3D_API int32_t m3d_gpu_autotune(m3d_world* world, int32_t stepsPerTrial);
M3D_API int32_t m3d_gpu_autotune_state(m3d_world* world, int32_t* tinyContacts, int32_t* tinyModeIslands);

/* Steps this world took through the sleeping-world fast path: when the
 * previous step changed nothing, every body was asleep before and after it
 * and no API call has edited the world since, m3d_world_step does on the
 * host what the reference's step does to such a world (advance the
 * stable-tier schedule, report the profile) and launches nothing. */
M3D_API int64_t m3d_gpu_fast_path_steps(m3d_world* world);

/* Failure handling (no counterpart in the reference).  Every device-side
 * wait of a step (the look-back of the scans, the grid barriers and the
 * colouring / overflow-level dataflow of the whole-GPU island solve) gives up
 * after a bounded number of unsuccessful polls and raises M3D_GPU_ERR_WAIT
 * instead of hanging.  A scan that gives up computes its prefix directly, so
 * the step's results stay exact; a giant-island solve that gives up stops at
 * its next grid barrier, leaving that island's substeps unfinished (the
 * world can be stepped on).  m3d_gpu_set_wait_limit sets the number of polls
 * (< 0: the defaults, about a second; 0: no scan waits at all and a barrier
 * gives up at its first unsuccessful poll) - a test aid for these paths.
 * m3d_gpu_clear_status resets the sticky status to M3D_GPU_OK. */
M3D_API void m3d_gpu_set_wait_limit(m3d_world* world, int64_t polls);
M3D_API void m3d_gpu_clear_status(m3d_world* world);

/* 0 when healthy, else the first M3D_GPU_ERR_* seen since creation. */
M3D_API int32_t m3d_gpu_status(m3d_world* world);
M3D_API const char* m3d_gpu_last_error_string(m3d_world* world);

/* Sphere cast that allocates nothing.  It has no counterpart in the
 * reference.  Same result as m3d_world_sphere_cast (melon3d.h), written to
 * *out; returns M3D_GPU_OK or an M3D_GPU_ERR_* code.
 *
 * Why: m3d_world_sphere_cast keeps one candidate record per body slot in a
 * device buffer that grows with the world, and first uploads any pending API
 * edits, which can grow other device buffers.  Callers that cannot allocate
 * device memory at query time need a path that never does: code that runs
 * under a fixed device-memory budget with the rest of HBM owned by another
 * allocator, and latency-critical callers (a frame's gameplay queries) for
 * which a cudaMalloc or cudaFree would stall on the device.  This entry point
 * uses one block of device memory built into the library (about 1.8 MB per
 * device) and calls no cudaMalloc, cudaFree or other allocating routine.
 *
 * Limits and rules:
 *  - worlds of at most 65536 body slots (m3d_gpu_body_capacity); larger ones
 *    are rejected with M3D_GPU_ERR_LIMIT and a message on stderr;
 *  - edits made through melon3d.h since the last step or query are not
 *    uploaded here: the call returns M3D_GPU_ERR_PENDING until the world is
 *    stepped or queried through m3d_world_* once;
 *  - the first call on a device looks up the block's device address
 *    (cudaGetSymbolAddress, with the world's device made current) and caches
 *    it with the device's current CUDA context; make that first call before
 *    any stream capture on that device.  If the context is later destroyed
 *    and recreated (cudaDeviceReset, or a framework resetting the primary
 *    context), the next call sees a different context and looks the address
 *    up again (again: not inside a stream capture);
 *  - the block is shared by every world and every call on the device and
 *    keeps the last call's contents (each call resets the parts it reads
 *    before use); each call waits for its own work, but calls whose work
 *    overlaps on the GPU (made at the same time from different host threads,
 *    for different worlds) race on the block: serialise them.
 * On M3D_GPU_ERR_* returns, *out (when non-NULL) holds a no-hit result. */
M3D_API int32_t m3d_gpu_sphere_cast_noalloc(m3d_world* world, m3d_vec3 origin, float radius, m3d_vec3 translation,
                                            uint32_t maskBits, m3d_ray_result* out);

/* Launch accounting (process-wide).  Every kernel launch of the library is
 * counted; the kernels named in m3d_gpu_profiler_reset (source names, e.g.
 * "kNarrowphase" or "kSolveSerial,kSolveFree"; "*" for every kernel; NULL for
 * none) are also bracketed by CUDA events on their stream, so their average
 * device duration can be read while the world runs.  m3d_gpu_profiler_table
 * writes one line per timed kernel, "<name> <launches> <total ms>", and
 * returns the table's full length. */
M3D_API void m3d_gpu_profiler_reset(const char* kernelName);
M3D_API long long m3d_gpu_profiler_launches(void);
M3D_API void m3d_gpu_profiler_kernel(float* totalMs, int32_t* launches);
M3D_API int32_t m3d_gpu_profiler_table(char* out, int32_t capacity);
/* Host->device and device->host bytes the library copied since the reset. */
M3D_API void m3d_gpu_profiler_bytes(long long* h2d, long long* d2h);
/* Device allocations (cudaMalloc calls) the library has made since it was
 * loaded (not reset by m3d_gpu_profiler_reset). */
M3D_API long long m3d_gpu_profiler_allocations(void);

/* ---- differentiation (no counterpart in the reference) ----------------------
 * m3d_gpu_tape_begin opens a tape: every following m3d_world_step records
 * what its adjoint needs (the contact set, solve order and manifolds of each
 * substep with their point ids and generation events, the islands, the
 * bodies put to sleep), and body states are checkpointed every
 * `checkpointEvery` steps (<= 0: 10).  m3d_gpu_step_backward then runs the
 * adjoint of all recorded steps on the device: given dL/d(final state) per
 * body slot, it returns dL/d(state at the tape's start) and dL/d(mass,
 * friction, restitution) per body slot.  The contact set, the solve order and
 * every branch the forward took are held fixed: the gradient is that of the
 * recorded branch.  Manifolds are differentiated as functions of the poses
 * they were generated at, and stiction anchors as state.  Covered: spheres
 * and boxes with isotropic inertia (cubes), free and contact-connected islands
 * below 300 contacts, no joints, no kinematic bodies, no applied forces, no
 * body edits between recorded steps.  Anything else marks the tape
 * unsupported (m3d_gpu_tape_supported) and the backward returns
 * M3D_GPU_ERR_UNSUPPORTED.
 *
 * Arrays are per body slot (m3d_gpu_body_capacity): positions and linear /
 * angular velocities 3 floats, rotations 4 (xyzw), scalars 1.  Input adjoint
 * arrays may be NULL (zero); output arrays may be NULL (not written). */
#define M3D_GPU_ERR_UNSUPPORTED (-8) /* the recorded steps use a feature the adjoint does not cover */
M3D_API int32_t m3d_gpu_tape_begin(m3d_world* world, int32_t checkpointEvery);
/* Discards the tape (recording stops). */
M3D_API void m3d_gpu_tape_end(m3d_world* world);
/* Steps recorded so far (0 without a tape). */
M3D_API int32_t m3d_gpu_tape_steps(m3d_world* world);
/* Device bytes the tape holds (contact records, island and body tables,
 * checkpoints); the backward reads all of them at least once. */
M3D_API int64_t m3d_gpu_tape_bytes(m3d_world* world);
/* Islands of the recorded steps that the replay and the backward work with a
 * whole warp each (islands with at least M3D_TAPE_WARP_CONTACTS contacts,
 * read from the environment when the tape opens; default 8, 0 = none); the
 * others take one thread each.  The results are the same either way. */
M3D_API int64_t m3d_gpu_tape_warp_islands(m3d_world* world);
/* 1 while the tape is differentiable; else 0 and the reason in why. */
M3D_API int32_t m3d_gpu_tape_supported(m3d_world* world, char* why, int32_t capacity);
/* Re-runs the recorded steps from the first checkpoint with the recorded
 * manifolds (the forward half of the adjoint) and returns the final states;
 * equal to the world's own states bit for bit. */
M3D_API int32_t m3d_gpu_tape_replay(m3d_world* world, float* positions, float* rotations, float* velocities,
								   float* angularVelocities, int32_t capacity);
M3D_API int32_t m3d_gpu_step_backward(m3d_world* world, const float* dPositions, const float* dRotations,
									  const float* dVelocities, const float* dAngularVelocities, float* gPositions,
									  float* gRotations, float* gVelocities, float* gAngularVelocities, float* gMass,
									  float* gFriction, float* gRestitution, int32_t capacity);
/* The same adjoint evaluated in double precision on the host from the same
 * tape: the FP64 reference gradient for checking m3d_gpu_step_backward. */
M3D_API int32_t m3d_gpu_step_backward_fp64_host(m3d_world* world, const double* dPositions,
												const double* dRotations, const double* dVelocities,
												const double* dAngularVelocities, double* gPositions,
												double* gRotations, double* gVelocities,
												double* gAngularVelocities, double* gMass, double* gFriction,
												double* gRestitution, int32_t capacity);
/* Verification aid: re-runs the recorded steps on the host from the first
 * checkpoint using only the tape's discrete record (islands, contact set,
 * solve order, generation events, sleeps) and regenerating every manifold
 * from the current poses at its recorded generation events.  In float
 * (doublePrecision 0) the result equals the world's own states bit for bit;
 * in double it is the function whose derivative m3d_gpu_step_backward
 * computes, for finite differences.  Perturbations, each NULL for none:
 * dVelocities and dAngularVelocities (3 per body slot) are added to the
 * initial velocities, dMass to the masses (inertia scaled along), dFriction
 * and dRestitution to the bodies' coefficients (contacts mix them as at their
 * creation). */
M3D_API int32_t m3d_gpu_tape_regenerate_host(m3d_world* world, int32_t doublePrecision, const double* dVelocities,
											 const double* dAngularVelocities, const double* dMass,
											 const double* dFriction, const double* dRestitution, double* positions,
											 double* rotations, double* velocities, double* angularVelocities,
											 int32_t capacity);

/* Snapshot records (melon3d_debug.h) — for tests and debugging. */
M3D_API int32_t m3d_dbg_body_capacity(m3d_world* world);
M3D_API void m3d_dbg_bodies(m3d_world* world, m3d_dbg_body* out, int32_t capacity);
M3D_API int32_t m3d_dbg_contact_count(m3d_world* world);
M3D_API void m3d_dbg_contacts(m3d_world* world, m3d_dbg_contact* out, int32_t capacity);
M3D_API void m3d_dbg_island_labels(m3d_world* world, int32_t* out, int32_t capacity);
M3D_API void m3d_dbg_contact_colors(m3d_world* world, int32_t* out, int32_t capacity);

#ifdef __cplusplus
}
#endif

#endif /* MELON3D_GPU_H */
