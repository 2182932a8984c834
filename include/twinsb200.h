/* twins-b200: the C ABI of the B200 packet-level simulator (libtwinsb200.so).
 *
 * The reference (TwiNS) exposes its TCP model only through the `twins` program: command-line
 * flags (src/main.cu:155-222), flow files (src/main.cu:110-137), topology files
 * (src/main.cu:227-252), worlds files (src/main.cu:283-325), and fct.csv
 * (src/main.cu:1143-1153); its device boundary is one Sim struct in constant memory and the
 * slot kernel ns_slot (src/kernel.cuh:5) captured into CUDA graphs (src/main.cu:1017-1049).
 * This header replaces that boundary with plain C entry points; the `twins` front-end
 * (twins_b200/csrc/twins_cli.cpp) reproduces the reference's command line over them.
 *
 * Conventions: every call returns an int status (TB_OK, a negative error, or TB_WARN_INEXACT);
 * tb_last_error() describes the last failure of the calling thread. The caller owns every host
 * buffer; the library owns device memory. No call exits the process. One context per host
 * thread.
 */
#ifndef TWINSB200_H
#define TWINSB200_H

#ifdef __cplusplus
extern "C" {
#endif

#define TB_OK 0
#define TB_WARN_INEXACT 1    /* a capacity overflowed or a tie was guessed: results may differ */
#define TB_ERR_ARG (-1)      /* a bad argument or input (bad flows, topology, world id) */
#define TB_ERR_CUDA (-2)     /* a CUDA call failed (no device, launch error) */
#define TB_ERR_MEMORY (-3)   /* the batch exceeds the context's HBM budget */
#define TB_ERR_STATE (-4)    /* a call out of order (e.g. results before a run) */
#define TB_ERR_TIMEOUT (-5)  /* a device-side wait ran out (the run was abandoned) */

#define TB_TOPO_FATTREE 0
#define TB_TOPO_LEAFSPINE 1
#define TB_TOPO_GRAPH 2

#define TB_TCP_NEWRENO 0
#define TB_TCP_DCTCP 1
#define TB_TCP_CUBIC 2

typedef struct tb_ctx tb_ctx;

/* A world's topology. Replaces --k / --topo=leafspine --leaves --spines --hpl /
 * --topo=graph --topofile --fail (reference src/main.cu:155-222, 223-465).
 * FatTree: k (a power of two, 4..32). Leaf-spine: leaves, spines, hpl (hosts per leaf).
 * Graph: n_hosts, n_switches and n_links links in file order, endpoints host h -> h and switch
 * j -> -1 - j (a host's one link has the host first); link failures at fail_t_ns[i] of the first
 * link between switches fail_a[i] and fail_b[i], down or (fail_up[i]) up again. */
typedef struct tb_topology
{
    int kind;
    int k;
    int leaves, spines, hpl;
    int n_hosts, n_switches, n_links;
    const int *link_a, *link_b;
    int n_fails;
    const long long *fail_t_ns;
    const int *fail_a, *fail_b, *fail_up;
} tb_topology;

/* A TCP world's parameters: --tcp --ecnK --queue --fin --spray --RngSeed --RngRun
 * (reference src/main.cu:155-222; per-world values as a worlds file gives them, :283-325). */
typedef struct tb_tcp_params
{
    int tcp;       /* TB_TCP_* */
    int ecn_k;     /* RED MinTh = MaxTh (packets), default 30 */
    int queue;     /* RED queue limit (packets), default 200 */
    int fin;       /* senders close after their last flow */
    int spray;     /* per-packet ECMP (MRG32k3a), else per-flow ECMP */
    unsigned rng_seed;
    unsigned long long rng_run;
} tb_tcp_params;

/* Run statistics of the last tb_run. */
typedef struct tb_stats
{
    long long slots;         /* the slot reached (simulated time in us) */
    long long slots_run;     /* slots executed (idle slots are skipped exactly) */
    long long launches;      /* persistent-kernel launches */
    double kernel_ms;        /* device time of the slot loop (CUDA events) */
    double upload_ms;        /* host-to-device time of the batch (tb_prepare) */
    unsigned long long packet_events; /* frame arrivals handled at hosts and switch ports */
    unsigned long long host_events, switch_events;
    unsigned long long host_sender_events; /* host arrivals handled by a connection's sender */
    unsigned long long host_frames;        /* frames hosts emitted */
    unsigned long long bytes_h2d, bytes_d2h;
    int grid, host_lanes, warps_per_block; /* the launch shape that ran the most slots */
    int stage_frames;        /* frames a warp stages in shared memory in that shape */
    int autotuned;           /* 1: the shape was picked per launch by measured throughput */
    int port_local;          /* 1: that shape keeps switch ports' slot state in shared memory */
    long long graph_launches; /* launches replayed from a captured CUDA graph */
} tb_stats;

/* A context on CUDA device `device`, admitting batches up to hbm_budget_bytes of device memory
 * (0: no limit). Replaces the reference's implicit device set-up (src/main.cu:51-58). Device -1
 * gives a host-only context: worlds can be added and their ECMP hashes read (tb_hashes), but
 * tb_prepare / tb_run fail with TB_ERR_STATE. */
int tb_ctx_create(int device, unsigned long long hbm_budget_bytes, tb_ctx **out);
int tb_ctx_destroy(tb_ctx *ctx);
const char *tb_last_error(void);

/* Adds one TCP world (one simulation) to the context's batch and returns its id in *world.
 * Flows are rows of a flow file (reference src/main.cu:110-137, 531-648): src, dst, size
 * (bytes), start_ns, and conn (NULL or -1: a connection of its own; rows with the same conn are
 * messages of one persistent connection, same hosts, later starts). hash_data / hash_ack: NULL
 * (the library computes ns-3's ECMP hashes, src/main.cu:674-723) or per-row hashes as
 * --ecmp_from takes them from an ns-3 output (src/main.cu:724-768). Worlds of one batch may
 * differ in topology and every parameter (the reference batches one topology only,
 * src/main.cu:267-270). */
int tb_world_add_tcp(tb_ctx *ctx, const tb_topology *topo, int n_flows, const int *src, const int *dst,
                     const long long *size, const long long *start_ns, const long long *conn,
                     const unsigned *hash_data, const unsigned *hash_ack, const tb_tcp_params *params, int *world);

/* Adds one RDMA world (the reference's twins-rdma model of the HPCC fork of ns-3.17: NICs with
 * queue pairs paced by rate, a window and go-back-N; switches with the PFC shared-buffer MMU and
 * ECN at dequeue; DCQCN, HPCC or DCTCP) and returns its id in *world. config: the HPCC config
 * file's "KEY VALUE" lines with any KEY=VALUE overrides applied (src/rdma/rmain.cu:100-143,
 * 364-527); topology: TwiNS's "hosts H / switches S / link A B" text (src/rdma/rmain.cu:471-520),
 * every link at link_bps with link_delay_ns; flows: rows of a flow file src,dst,flow_size,start_ns
 * (src/rdma/rmain.cu:842-1021). A context holds TCP worlds or RDMA worlds, not both (TB_ERR_STATE);
 * RDMA worlds of one context run side by side in one launch, as the reference's --batch
 * (src/rdma/rmain.cu:1204-1362). Refusals the reference makes return TB_ERR_ARG with its reason. */
int tb_world_add_rdma(tb_ctx *ctx, const char *config, const char *topology, int n_flows, const int *src, const int *dst,
                      const long long *size, const long long *start_ns, unsigned long long link_bps, long long link_delay_ns,
                      int *world);
/* After tb_run of RDMA worlds: per flow (in file order) its start and completion time minus start
 * (ns; -1: not done), as the reference's "id start_ns fct_ns" output (src/rdma/rmain.cu:2178-2200).
 * tb_counters gives the run's 40 counters in the reference's order (src/rdma/rmain.cu:2239-2261:
 * drops, marks, pauses, resumes, tx / queue / ackq / qps overflows, undecided ties, lost tails, ACKs
 * for done QPs, NACKs, due overflow, late data); tb_run returns TB_WARN_INEXACT where the reference
 * exits 3. */
int tb_rdma_results(tb_ctx *ctx, int world, long long *start_ns, long long *fct_ns);
/* Frames a switch port's data queue holds in this context's RDMA run (default 4096, as the
 * reference's --q3cap, src/rdma/rmain.cu:1054, 1811); a frame that finds it full is counted as an
 * overflow (the run is then inexact). Before the first run. */
int tb_rdma_set_queue_cap(tb_ctx *ctx, int frames);
/* A transmission of an RDMA run as the reference's --txtrace records it (src/rdma/rdma.h TxRec,
 * written by src/rdma/rmain.cu:2262-2282): its start (ns), the ns-3 node (hosts, then switches)
 * and device (a host's NIC 1, switch port p + 1), the kind (0 data, 1 ACK, 2 NACK, 3 PAUSE, 4
 * RESUME; "DANPR"), a / b the flow's hosts as the sender sees them (data: source, destination;
 * ACK / NACK: destination, source; PFC: the queue, 0), the source port, sequence, bytes and ECN. */
typedef struct tb_tx_record
{
    long long ts_ns;
    int node, dev;
    unsigned a, b, sport, seq;
    unsigned short size;
    unsigned char kind, ecn;
} tb_tx_record;
/* Before the first run of a context with ONE RDMA world: keep up to `cap` transmission records of
 * frames that start in [from_ns, until_ns] (the reference's --txtrace=F --from=ns --until=ns; it
 * refuses a batch too). cap 0 turns the trace off. */
int tb_rdma_set_txtrace(tb_ctx *ctx, long long cap, long long from_ns, long long until_ns);
/* After the run: the records sorted by (start, node, device), up to `cap` of them into `out`;
 * *n the records written, *total the transmissions in the window (more than kept when the trace's
 * cap was reached, as the reference's "txtrace: N records, M kept"). */
int tb_rdma_txtrace(tb_ctx *ctx, tb_tx_record *out, long long cap, long long *n, long long *total);

/* Builds the batch's device state (routes, connections, rings) and uploads it. Called by
 * tb_run when needed; separate so that timing can exclude it. Replaces src/main.cu:807-1015. */
int tb_prepare(tb_ctx *ctx);

/* Restores every world of the prepared batch to its initial state (device-to-device). */
int tb_reset(tb_ctx *ctx);

/* Runs every world of the batch until all of its flows complete or max_slots slots (1 us each)
 * have passed (0: the reference's default, 2,000,000). Replaces the graph loop of
 * src/main.cu:1017-1049 and the slot kernel src/kernel.cuh:5-113. Returns TB_WARN_INEXACT if a
 * capacity overflowed or an event-order tie was guessed (reference warnings, src/main.cu:1070-1075). */
int tb_run(tb_ctx *ctx, long long max_slots);

/* Per flow row (file order) of a world: established_ns and completed_ns (-1: not reached), the
 * columns of fct.csv (src/main.cu:1143-1153). */
int tb_results(tb_ctx *ctx, int world, long long *established_ns, long long *completed_ns);

/* Counters of a world (n <= 16): drops, marks, retransmissions, RTOs, undecided ties, host
 * packet-events, switch packet-events, overflow counts (active lists, timers, rings,
 * out-of-order blocks, tx-cap), barrier timeouts, sender-side host packet-events, frames hosts
 * emitted (reference counters, src/main.cu:1064-1075). */
int tb_counters(tb_ctx *ctx, int world, unsigned long long *out, int n);

/* Per flow row of a world: the ECMP hashes in use (reference --hash_check, src/main.cu:755-768). */
int tb_hashes(tb_ctx *ctx, int world, unsigned *hash_data, unsigned *hash_ack);

/* Statistics of the last run. */
int tb_get_stats(tb_ctx *ctx, tb_stats *out);

/* Launch shape: hosts per warp (1..32) and the grid (0: chosen from occupancy); turns autotuning
 * off. Replaces the reference's --host_lanes (src/main.cu:183-184, 523-526). */
int tb_set_launch(tb_ctx *ctx, int host_lanes, int grid);
/* The same with the frames a warp stages in shared memory per slot (1..384, 1..256 in the 25-run
 * build; default 192; fewer leave room for more resident blocks per SM, more stage the slots of
 * big switches). */
int tb_set_launch_shape(tb_ctx *ctx, int host_lanes, int stage_frames, int grid);
/* A fixed shape's switch egress (one host per warp only): 1 keeps each port's transmission chain
 * and last enqueued frame in shared memory for the slot (faster where big switches are the
 * critical path), 0 (default) reads them from the port's record. Autotuning picks it per launch. */
int tb_set_port_local(tb_ctx *ctx, int on);
/* Autotuning (on by default): tb_run picks each launch's shape (hosts per warp, staging size)
 * among a fixed set by the packet-events per ms that short probe launches of each achieve. The
 * results never depend on the shape (no counterpart in the reference). */
int tb_set_autotune(tb_ctx *ctx, int on);
/* Batches (on by default): 1 runs each world of a batch on a barrier of its own, so that a world's
 * slot waits only for that world's units (the reference's batch launch, src/main.cu:267-325, keeps
 * every world of the batch in the same slot); 0 keeps one grid-wide barrier per slot. The results
 * never depend on it (no counterpart in the reference). */
int tb_set_free_batches(tb_ctx *ctx, int on);

/* sizeof(tb_topology), sizeof(tb_tcp_params), sizeof(tb_stats), sizeof(tb_serve_caps),
 * sizeof(tb_request_info), sizeof(tb_serve_stats), sizeof(tb_qrec), sizeof(tb_tx_record) in
 * out[0..n-1], so that
 * bindings in other languages can check their struct layouts (no counterpart in the reference). */
int tb_abi_sizes(unsigned long long *out, int n);

/* One TCP world run to completion without allocating device memory (no counterpart in the
 * reference). For callers that cannot call cudaMalloc: a process whose device memory belongs to
 * a framework's caching pool, code that must not allocate while it runs, or a process under a
 * hard memory cap. The world's whole device state is carved from a fixed 48 MiB area that every
 * process loading the library holds on each device it uses until it exits; a world that needs
 * more (e.g. a FatTree k=8) is rejected with TB_ERR_MEMORY before anything runs. Arguments are
 * tb_world_add_tcp's and tb_run's (ECMP hashes computed), results as tb_results gives them into
 * the caller's host arrays. Each call looks up the area's device address with that device
 * current (the first call on a device loads the module there, so make it before any stream
 * capture). Every call on a device shares the area, which keeps the last call's contents; each
 * call clears what must start at zero. Calls that overlapped on the GPU would race on the area,
 * so the library makes the calls of one process take turns (a lock held for the whole call).
 * The call runs its copies and launches on the legacy default stream and returns when they are
 * done: it waits for earlier work on the caller's blocking streams (as that stream does), but
 * not for non-blocking streams, and it does not synchronize the whole device. */
int tb_run_static(int device, const tb_topology *topo, int n_flows, const int *src, const int *dst,
                  const long long *size, const long long *start_ns, const long long *conn,
                  const tb_tcp_params *params, long long max_slots, long long *established_ns,
                  long long *completed_ns);

/* ---- the enqueue trace (the reference's --qtrace, src/main.cu:169-174, 985-994, 1077-1100;
 * record src/model.h:313-320): every packet a queue accepts with from_ps <= its time < until_ps.
 * Recorded only by the trace build (libtwinsb200_trace.so, front-end twins-trace); the others
 * return TB_ERR_STATE. */
typedef struct tb_qrec
{
    long long ts;                /* ps */
    int node, dev, src, dst;     /* ns-3 node (hosts, then switches) and device (NIC 1, port p+1) */
    unsigned sa;                 /* sequence (data) or acknowledgement number */
    unsigned short len, qlen;    /* bytes on the wire; the queue disc's length after the enqueue */
    unsigned char flags, pad[3];
} tb_qrec;

int tb_has_qtrace(void);
int tb_set_qtrace(tb_ctx *ctx, unsigned long long capacity, long long from_ps, long long until_ps);
/* After tb_run: the records (in recording order, at most cap), *n the number recorded (<= capacity). */
int tb_qtrace(tb_ctx *ctx, tb_qrec *out, unsigned long long cap, unsigned long long *n);

/* ---- serving: requests join a running batch (no counterpart in the reference, which runs one
 * batch fixed at start, src/main.cu:283-325). A server holds device arrays sized by its
 * capacities and runs the slot kernel over them in launches of slots_per_launch slots; between
 * launches it retires finished worlds and admits queued requests into free room, each starting
 * its own time at the launch slot it joins, so its results equal a standalone run's. */
typedef struct tb_server tb_server;

typedef struct tb_serve_caps
{
    int worlds;                           /* requests in the batch at once */
    int hosts, switches, ports;           /* entities over all requests in the batch */
    int connections, messages;
    unsigned long long sent_list_entries; /* per-connection sent-list / RTT-history ring entries */
    unsigned long long ooo_blocks;        /* receivers' out-of-order block entries */
    int active_per_host;                  /* connections one host holds on one side */
    int max_queue;                        /* the largest RED queue limit a request may set */
    int max_ports;                        /* ports per switch, <= 32 */
    int slots_per_launch;                 /* admission granularity (slots of 1 us) */
    unsigned long long hbm_budget_bytes;  /* 0: no limit */
} tb_serve_caps;

typedef struct tb_request_info
{
    int state;            /* 0 queued, 1 running, 2 done, 3 failed */
    int n_flows;
    double t_submit, t_admit, t_done; /* seconds, the server's steady clock */
    long long slot0, slots;          /* the launch slot it joined, the slots it took */
} tb_request_info;

typedef struct tb_serve_stats
{
    long long launches, slots_run, admitted, retired, queued, running;
    double kernel_ms;                 /* device time of all launches */
    unsigned long long packet_events, hbm_bytes;
    int host_lanes, stage_frames, grid;
} tb_serve_stats;

int tb_server_create(int device, const tb_serve_caps *caps, tb_server **out);
int tb_server_destroy(tb_server *srv);
/* Queues a TCP world (the arguments of tb_world_add_tcp without given hashes); thread-safe.
 * Fails with TB_ERR_MEMORY if the request could never fit the server's capacities. */
int tb_server_submit_tcp(tb_server *srv, const tb_topology *topo, int n_flows, const int *src, const int *dst,
                         const long long *size, const long long *start_ns, const long long *conn,
                         const tb_tcp_params *params, long long *request);
/* One round on the calling thread: admit, run one launch, retire. *running: requests in the
 * batch afterwards. Not with tb_server_start. */
int tb_server_step(tb_server *srv, int *running);
/* Runs the rounds on a thread of the server's own while requests are queued or running. */
int tb_server_start(tb_server *srv);
/* Blocks until the request is done (timeout_s <= 0: no limit). */
int tb_server_wait(tb_server *srv, long long request, double timeout_s);
/* A done request's results (as tb_results / tb_counters, rows in submission order) and its
 * timeline; any output may be NULL (info alone also works before it is done). */
int tb_server_results(tb_server *srv, long long request, long long *established_ns, long long *completed_ns,
                      unsigned long long *counters, int n_counters, tb_request_info *info);
/* Forgets a queued or done request. */
int tb_server_release(tb_server *srv, long long request);
int tb_server_stats(tb_server *srv, tb_serve_stats *out);

#ifdef __cplusplus
}
#endif

#endif
