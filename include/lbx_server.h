/* lbx_server.h -- native continuous-batching request loop over the ensemble engine.
 *
 * No counterpart in the reference, which solves one SuperLattice per program run
 * (examples/laminar/cavity3dBenchmark/cavity3d.cpp:189-233 and :241 -- set up, step, evaluate -- is
 * the plain solve that a parameter sweep repeats).  The server takes parameter-sweep requests (lbx_ensemble_request: a box cavity
 * of its own size and Reynolds number) from any host thread, and one host thread of its own
 * runs the loop:
 *
 *   1. requests whose arrival time has come join the waiting queue (in arrival order);
 *   2. every waiting request whose slab footprint fits is admitted as a slot (first fit: one
 *      that does not fit yet does not hold back smaller ones behind it);
 *   3. all admitted lattices are stepped together by one ensemble run of `chunk` steps;
 *   4. every slot the engine reports converged, capped or diverged is retired at once, its
 *      memory freed for the queue, and its record (arrival, admission and finish times, steps,
 *      state, residual) made available to lbx_server_records.
 *
 * Requests that arrive while others are on the GPU join at the next run boundary.  The chunk
 * adapts: `min_chunk` steps while a request waits for memory or one is due to arrive within the
 * next long run, `max_chunk` steps otherwise (both are replayed from CUDA graphs the engine keeps
 * per step count).  Times are seconds after lbx_server_start, on the wall clock (realtime = 1)
 * or on a virtual clock that advances by the measured duration of each run and jumps over idle
 * gaps to the next arrival (realtime = 0: a recorded arrival trace replayed as fast as the GPU
 * serves it).
 *
 * The loop drives the engine through lbx_server_engine, so an embedding can put its own engine
 * behind it (the tests drive the loop with a host-side fake engine); lbx_server_create binds an
 * lbx_ensemble.  Every call returns 0 or a negative lbx_status (lbx.h); lbx_last_error() gives
 * the message of a failure on the calling thread. */
#ifndef LBX_SERVER_H
#define LBX_SERVER_H

#include "lbx.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lbx_server_s* lbx_server;

/* Record states beyond lbx_slot_state. */
enum {
  LBX_SERVER_REJECTED = 5,   /* the engine refused the request (invalid, or larger than an empty engine) */
  LBX_SERVER_CANCELLED = 6   /* lbx_server_cancel before it finished */
};

typedef struct {
  int64_t id;                   /* the caller's request id (reported back in the record) */
  double arrival;               /* seconds after lbx_server_start; < 0: the time of submission */
  lbx_ensemble_request request;
} lbx_server_request;

typedef struct {
  int64_t id;
  int64_t cells;                /* core cells of the request */
  double arrival, admitted, finished;  /* seconds after lbx_server_start (NaN: never admitted) */
  int64_t steps;                /* steps taken */
  int32_t state;                /* lbx_slot_state (CONVERGED, MAX_STEPS, DIVERGED) or LBX_SERVER_* */
  int32_t slot;                 /* the engine slot it ran in (-1: never admitted) */
  double residual;              /* last checked residual */
} lbx_server_record;

typedef struct {
  int32_t min_chunk;   /* steps per run while a request waits or is due (>= 1) */
  int32_t max_chunk;   /* steps per run otherwise (>= min_chunk) */
  int32_t realtime;    /* 1: wall clock; 0: virtual clock (see above) */
  int32_t pad;
} lbx_server_config;

/* The engine behind the loop.  admit returns 0 and the slot, LBX_ERR_OUT_OF_MEMORY when the
 * request does not fit yet, or another negative status to reject it; run steps every admitted
 * lattice; statuses fills `slots` entries; retire frees a slot.  All are called from the loop's
 * own thread only. */
typedef struct {
  int32_t (*admit)(void* ctx, const lbx_ensemble_request* req, int32_t* slot);
  int32_t (*run)(void* ctx, int32_t steps);
  int32_t (*statuses)(void* ctx, lbx_ensemble_status* out, int32_t n);
  int32_t (*retire)(void* ctx, int32_t slot);
  int32_t slots;       /* number of slot entries statuses reports */
  int32_t pad;
} lbx_server_engine;

/* A server over an ensemble with `max_lattices` slots (as created), its work ordered on
 * `stream`.  The ensemble must not be used by anything else while the loop runs. */
int lbx_server_create(lbx_ensemble ens, int32_t max_lattices, const lbx_server_config* cfg, void* stream,
                      lbx_server* out);
/* A server over a caller-supplied engine (`engine` is copied; `ctx` is passed to its calls). */
int lbx_server_create_with_engine(const lbx_server_engine* engine, void* ctx, const lbx_server_config* cfg,
                                  lbx_server* out);
/* Called on the loop's thread for every record as it is made, before the slot is retired (the
 * slot's fields can still be read, e.g. with lbx_ensemble_moments). */
typedef void (*lbx_server_finish_fn)(void* user, const lbx_server_record* record);
int lbx_server_set_finish_callback(lbx_server s, lbx_server_finish_fn fn, void* user);
/* Queue requests (any thread, before or after start).  LBX_ERR_INVALID after lbx_server_close. */
int lbx_server_submit(lbx_server s, const lbx_server_request* requests, int32_t n);
/* Start the loop on its own thread; the clock starts here. */
int lbx_server_start(lbx_server s);
/* No more submissions: the loop ends once every submitted request has a record. */
int lbx_server_close(lbx_server s);
/* Cancel a request by id: a waiting one is dropped, a running one retired at the next run
 * boundary; both get a record with state LBX_SERVER_CANCELLED.  LBX_ERR_INVALID if the id is not
 * waiting or running. */
int lbx_server_cancel(lbx_server s, int64_t id);
/* Wait up to timeout_s seconds (< 0: no limit) for the loop to end.  *finished = 1 when it has
 * ended; the return value is then the loop's own status (0, or the engine error that stopped it). */
int lbx_server_wait(lbx_server s, double timeout_s, int32_t* finished);
/* Take up to `capacity` finished records (oldest first); *n_out = how many were written. */
int lbx_server_records(lbx_server s, lbx_server_record* out, int32_t capacity, int32_t* n_out);

typedef struct {
  int64_t submitted, pending, waiting, running, finished;  /* requests by where they are */
  int64_t runs, steps;            /* engine runs made and steps they took */
  int64_t short_runs, long_runs;  /* runs of min_chunk and of max_chunk steps */
  double busy_seconds;            /* time inside engine runs and status reads */
  double clock;                   /* the server clock now (seconds after start) */
} lbx_server_stats;
int lbx_server_get_stats(lbx_server s, lbx_server_stats* out);
/* Stop the loop after its current run (if running) and free the server; records not taken are
 * lost.  Slots still admitted are retired. */
int lbx_server_destroy(lbx_server s);

#ifdef __cplusplus
}
#endif

#endif /* LBX_SERVER_H */
