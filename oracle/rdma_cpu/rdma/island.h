// Test infrastructure, not product code: the reference's twins-rdma run on the CPU.
//
// `make -C oracle ref-rdma-cpu` builds the reference's own src/rdma/rmain.cu with g++ under its
// TWINS_CPU shim (src/gpu_runtime.h: device memory is host memory, one lane per block) and
// TWINS_ISLAND, whose hooks rmain.cu takes from "rdma/island.h". This file stands in for the
// reference's island.h (found first on the include path): its hooks leave the worlds as rmain.cu
// builds them (plain flows, no DAG messages from outside), and island_run steps every block of
// every slot in turn, as the GPU's launches would, until the run finishes. The result is the
// reference's twins-rdma, with its command line, files and output, as a CPU program: the oracle
// for RDMA worlds where no GPU is at hand. Worlds with wide switches (which the GPU runs in
// rdma_slot_big's blocks) are refused.
#pragma once
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

static std::string g_isl_in, g_isl_map, g_isl_out, g_isl_shm, g_isl_rings;
static int g_isl_side = 0, g_isl_nrings = 0, g_isl_ringlog = 22;

namespace rdma
{
// (every tail node is this process's own)
uint64_t g_tail_side = 0;
TailNode island_remote(uint64_t) { return TailNode{}; }
} // namespace rdma

static void island_world(World &) {}
static void island_setup(Sim &) {}

static void island_run(Sim &s, int64_t)
{
    if (s.ns_b > 0)
    {
        fprintf(stderr, "rdma-cpu: %d wide switches: not run on the CPU\n", s.ns_b);
        exit(3);
    }
    blockDim.x = 1;
    threadIdx.x = 0;
    std::vector<char> smem(1 << 22);
    const int nb = s.n1 + s.ns_s + s.nm;
    while (!*s.finished)
    {
        const int64_t slot = *s.slot;
        for (int b = 0; b < nb; b++)
        {
            blockIdx.x = b;
            slot_entity<false>(s, b, s.bi_s[b], slot, smem.data(), 1);
        }
    }
}
