/* numa_shim.c (oracle shim, TEST INFRASTRUCTURE): an empty run-node mask, so the
 * reference's NUMA binding loop (grainhdl.cpp:1338-1388) binds nothing. */
#include "numa.h"
#include <stdlib.h>

static unsigned long g_empty_bits[1];
static struct bitmask g_empty = {0, g_empty_bits};
struct bitmask* numa_all_cpus_ptr = &g_empty;

int numa_available(void) { return -1; }
struct bitmask* numa_get_run_node_mask(void) { return &g_empty; }
struct bitmask* numa_allocate_cpumask(void) {
    struct bitmask* b = (struct bitmask*)calloc(1, sizeof(*b));
    b->maskp = (unsigned long*)calloc(1, sizeof(unsigned long));
    return b;
}
void numa_free_cpumask(struct bitmask* b) { if (b) { free(b->maskp); free(b); } }
int numa_bitmask_isbitset(const struct bitmask* b, unsigned int n) {
    return b && n < b->size && ((b->maskp[n / (8 * sizeof(unsigned long))] >> (n % (8 * sizeof(unsigned long)))) & 1ul);
}
int numa_node_to_cpus(int node, struct bitmask* mask) { (void)node; (void)mask; return -1; }
