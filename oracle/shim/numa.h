/*
 * Test-infrastructure shim (oracle only): the libnuma calls made by
 * GraGLeS2D's thread binding (src/grainhdl.cpp:1529-1591).  libnuma is not
 * installed; the shim reports no NUMA node, so the reference binds no thread
 * and runs its OpenMP regions unpinned.
 */
#ifndef GG_ORACLE_NUMA_SHIM_H
#define GG_ORACLE_NUMA_SHIM_H
#ifdef __cplusplus
extern "C" {
#endif
struct bitmask {
    unsigned long size;
    unsigned long* maskp;
};
extern struct bitmask* numa_all_cpus_ptr;
int numa_available(void);
struct bitmask* numa_get_run_node_mask(void);
struct bitmask* numa_allocate_cpumask(void);
void numa_free_cpumask(struct bitmask* b);
int numa_bitmask_isbitset(const struct bitmask* b, unsigned int n);
int numa_node_to_cpus(int node, struct bitmask* b);
#ifdef __cplusplus
}
#endif
#endif
