/* Stand-in for the external emu_c_utils library (not shipped with the
 * reference).  Test infrastructure only.
 *
 * It supplies what the reference's x86 build takes from emu_c_utils:
 *   - the memoryweb intrinsics, by including the reference's own x86 shim
 *     emu_cxx_utils/memoryweb_x86.h (found on the include path);
 *   - the hooks_* timing API used by hybrid_bfs_main.cc:150-174,266-282 and
 *     graph_base.h:358-428.  hooks_region_end() returns the elapsed
 *     milliseconds of the innermost open region, which is how
 *     hybrid_bfs_main.cc:282 reads the BFS time.
 */
#pragma once
#include <emu_cxx_utils/memoryweb_x86.h>
#include <assert.h>
#include <time.h>

#ifdef __cplusplus
extern "C" {
#endif

static inline double bd_stub_now_ms(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec * 1e3 + (double)ts.tv_nsec * 1e-6;
}

/* A small stack of open regions; regions nest at most a few deep. */
static double bd_stub_region_start[64];
static int bd_stub_region_depth = 0;

static inline void hooks_set_active_region(const char *name) { (void)name; }
static inline void hooks_set_attr_i64(const char *key, long value) { (void)key; (void)value; }
static inline void hooks_set_attr_str(const char *key, const char *value) { (void)key; (void)value; }
static inline void hooks_region_begin(const char *name)
{
    (void)name;
    if (bd_stub_region_depth < 64) {
        bd_stub_region_start[bd_stub_region_depth] = bd_stub_now_ms();
    }
    ++bd_stub_region_depth;
}
static inline double hooks_region_end(void)
{
    if (bd_stub_region_depth <= 0) { return 0.0; }
    --bd_stub_region_depth;
    if (bd_stub_region_depth >= 64) { return 0.0; }
    return bd_stub_now_ms() - bd_stub_region_start[bd_stub_region_depth];
}

#ifdef __cplusplus
}
#endif
