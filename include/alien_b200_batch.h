/*
 * alien_b200_batch.h - batched multi-world stepping on one GPU.
 *
 * No counterpart in the reference: its facade owns exactly one world
 * (_SimulationCudaFacade, source/EngineGpuKernels/SimulationCudaFacade.cuh
 * :27-139).  A batch holds many independent worlds of different sizes and
 * parameters in one device arena; one timestep of all of them is one launch
 * per phase, replayed from a CUDA graph.  Each world evolves exactly as it
 * would alone in an alien_b200_simulation (same deterministic step).
 */
#ifndef ALIEN_B200_BATCH_H
#define ALIEN_B200_BATCH_H

#include "alien_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct alien_b200_batch alien_b200_batch;

/* general[w], params[w], data[w] describe world w (0 <= w < numWorlds). */
int alien_b200_batch_create(int numWorlds, const AlienGeneralSettings* general, const AlienPhysicsParams* params,
                            const AlienDataTO* data, uint64_t timestep, alien_b200_batch** out);
int alien_b200_batch_destroy(alien_b200_batch* batch);
int alien_b200_batch_num_worlds(alien_b200_batch* batch);
/* steps every world `timesteps` times and synchronises */
int alien_b200_batch_calc_timesteps(alien_b200_batch* batch, uint64_t timesteps);
/* enqueues the steps on the batch's stream without synchronising */
int alien_b200_batch_enqueue_timesteps(alien_b200_batch* batch, uint64_t timesteps);
/* waits for the enqueued steps, then grows particle storage where a world
 * has filled half of it (calc_timesteps does this every 64 steps); call it
 * at least every 64 enqueued steps.  A world whose step created more
 * particles than its range holds halted in that step; the wait grows its
 * range, completes the step and runs the steps it missed (the other worlds
 * parked), so every world ends as if its storage had been large enough.
 * ALIEN_B200_ERR_CAPACITY: a live arena had no larger free range for such a
 * world, whose steps then dropped the excess until the next capacity check
 * (the world still completed its steps). */
int alien_b200_batch_synchronize(alien_b200_batch* batch);
int alien_b200_batch_get_data(alien_b200_batch* batch, int world, const AlienDataTO* data);
int alien_b200_batch_get_array_sizes(alien_b200_batch* batch, int world, AlienArraySizes* sizes);
int alien_b200_batch_get_raw_statistics(alien_b200_batch* batch, int world, AlienRawStatistics* statistics);
int alien_b200_batch_get_raw_statistics_data(alien_b200_batch* batch, int world, AlienRawStatisticsData* statistics);
/* world's density map (alien_b200_get_density_map) */
int alien_b200_batch_get_density_map(alien_b200_batch* batch, int world, AlienDensityMap* map);
int alien_b200_batch_reset_time_interval_statistics(alien_b200_batch* batch, int world);
/* World `world` steps `steps` more times and then stops (its state stays
 * resident and readable); 0 = no limit.  Worlds start active, unlimited. */
int alien_b200_batch_set_step_budget(alien_b200_batch* batch, int world, uint64_t steps);
int alien_b200_batch_world_status(alien_b200_batch* batch, int world, uint64_t* timestep, uint64_t* stepsRemaining,
                                  int* active);
/* number of worlds still stepping (-1 on error) */
int alien_b200_batch_num_active(alien_b200_batch* batch);
/* device memory held by the batch's arena */
uint64_t alien_b200_batch_device_bytes(alien_b200_batch* batch);
void* alien_b200_batch_stream(alien_b200_batch* batch);
uint64_t alien_b200_batch_kernel_launch_count(alien_b200_batch* batch);
int alien_b200_batch_kernels_per_step(alien_b200_batch* batch);
/* event-timed steps as alien_b200_time_timesteps, for all worlds */
int alien_b200_batch_time_timesteps(alien_b200_batch* batch, uint64_t timesteps, double* milliseconds);
/* per-kernel timing as alien_b200_timed_timesteps, for all worlds */
int alien_b200_batch_timed_timesteps(alien_b200_batch* batch, uint64_t timesteps, double* kernelMs, int maxKernels,
                                     int* numKernels);
/* launch configuration of the batch's pair kernels (alien_b200_set_launch_config) */
int alien_b200_batch_set_launch_config(alien_b200_batch* batch, const AlienLaunchConfig* config);
int alien_b200_batch_get_launch_config(alien_b200_batch* batch, AlienLaunchConfig* config);

/*
 * Live arenas: worlds admitted and evicted while the others step.
 *
 * No counterpart in the reference (its EngineWorker, source/EngineImpl/
 * EngineWorker.cpp:450-476, steps one world).  A live arena reserves device
 * memory for a stated capacity once.  alien_b200_world_admit places a world
 * into free ranges of it and uploads and ingests the world on the arena's
 * stream, behind the steps already enqueued, without touching the other
 * worlds' state; alien_b200_world_evict frees a world's ranges.  Every
 * resident world steps in the same launches (alien_b200_batch_enqueue_timesteps
 * / calc_timesteps), and each evolves exactly as it would alone.  A live arena
 * is an alien_b200_batch: the world index returned by the admission is what
 * every alien_b200_batch_* call with a `world` argument takes (get_data,
 * statistics, step budget, status); alien_b200_batch_destroy releases it.
 * A world evicted or never admitted is an invalid index.
 */
typedef struct {
    int maxWorlds;              /* resident worlds at most (1 .. 65534) */
    uint64_t cellSlots;         /* cell slots: a world takes its cell count rounded up to 256 */
    uint64_t particleSlots;     /* particle slots: a world takes cells + particles + max(4096, (cells + particles) / 2),
                                   rounded up to 256 */
    uint64_t tiles;             /* hash tiles: a world of W x H slots takes ceil(W / r) * ceil(H / r), r = its
                                   interaction radius in whole slots (2 for the default parameters) */
    uint64_t particleMapSlots;  /* particle-map slots: a world takes W * H */
    uint64_t auxBytes;          /* auxiliary data (neuron weights and biases) */
} AlienArenaCapacity;

/* device bytes a live arena of this capacity reserves */
int alien_b200_arena_bytes(const AlienArenaCapacity* capacity, uint64_t* bytes);
int alien_b200_arena_create(const AlienArenaCapacity* capacity, alien_b200_batch** out);
/* Admits a world that steps `steps` times (0 = no limit) from `timestep`.
 * Returns ALIEN_B200_ERR_CAPACITY, with the arena unchanged, when a range or
 * a world slot is not free; the objects are validated as by set_data. */
int alien_b200_world_admit(alien_b200_batch* arena, const AlienGeneralSettings* general, const AlienPhysicsParams* params,
                           const AlienDataTO* data, uint64_t timestep, uint64_t steps, int* world);
/* Frees a resident world's ranges (read its results first). */
int alien_b200_world_evict(alien_b200_batch* arena, int world);
/* resident worlds of a live arena (-1 on error) */
int alien_b200_arena_num_resident(alien_b200_batch* arena);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* ALIEN_B200_BATCH_H */
