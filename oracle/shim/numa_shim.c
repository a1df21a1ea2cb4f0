/* Test-infrastructure shim (oracle only): single-node, no-binding libnuma. */
#include "numa.h"
#include <stdlib.h>

static struct bitmask empty_mask = {0, 0};
struct bitmask* numa_all_cpus_ptr = &empty_mask;

int numa_available(void) { return 0; }
struct bitmask* numa_get_run_node_mask(void) { return &empty_mask; }
struct bitmask* numa_allocate_cpumask(void) {
    struct bitmask* b = (struct bitmask*)calloc(1, sizeof(*b));
    return b;
}
void numa_free_cpumask(struct bitmask* b) { free(b); }
int numa_bitmask_isbitset(const struct bitmask* b, unsigned int n) {
    if (!b || n >= b->size || !b->maskp) return 0;
    return (int)((b->maskp[n / (8 * sizeof(unsigned long))] >> (n % (8 * sizeof(unsigned long)))) & 1UL);
}
int numa_node_to_cpus(int node, struct bitmask* b) {
    (void)node;
    (void)b;
    return 0;
}
