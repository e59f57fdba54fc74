/* numa.h (oracle shim, TEST INFRASTRUCTURE): the libnuma calls that
 * grainhdl::initNUMABindings (grainhdl.cpp:1338-1388) makes.  The run-node mask
 * is empty, so the reference pins no thread; pinning is left to OMP_PLACES. */
#ifndef GG_SHIM_NUMA_H
#define GG_SHIM_NUMA_H
#ifdef __cplusplus
extern "C" {
#endif
struct bitmask { unsigned long size; unsigned long* maskp; };
extern struct bitmask* numa_all_cpus_ptr;
int numa_available(void);
struct bitmask* numa_get_run_node_mask(void);
struct bitmask* numa_allocate_cpumask(void);
void numa_free_cpumask(struct bitmask* b);
int numa_bitmask_isbitset(const struct bitmask* b, unsigned int n);
int numa_node_to_cpus(int node, struct bitmask* mask);
#ifdef __cplusplus
}
#endif
#endif
