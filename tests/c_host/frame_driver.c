/* A native host of libfluidcu in plain C: what a C, Rust (bindgen), Go (cgo)
 * or Swift host links against in place of the reference's fluid_renderer_*
 * entry points. It creates the reference's test box, runs `frames` 1/120 s
 * frames under gravity (substeps chosen by the library from the last frame's
 * v_max, cap 16, seed = frame index), reads the statistics and the particles
 * back and destroys the simulation.
 *
 *     frame_driver [frames [particles.bin]]
 *
 * Prints one line: particle count, substeps run, the mean compression and
 * v_max as float bit patterns. With a file name it also writes the particles
 * there, positions (n x 4 floats) then velocities (n x 4 floats), in id
 * order. Exits 0; on a failure it prints fluid_last_error() to stderr and
 * exits 1.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fluid_cu.h"

static uint32_t bits(float v) {
    uint32_t u;
    memcpy(&u, &v, sizeof u);
    return u;
}

static int fail(const char *what, int32_t rc) {
    fprintf(stderr, "%s: status %d: %s\n", what, (int)rc, fluid_last_error());
    return 1;
}

int main(int argc, char **argv) {
    const int frames = argc > 1 ? atoi(argv[1]) : 30;
    FluidSimConfig cfg;
    fluid_sim_default_config(&cfg);
    FluidSim *sim = fluid_sim_create(&cfg);
    if (!sim) return fail("fluid_sim_create", -1);
    const FluidVec3 gravity = {0.0f, -9.81f, 0.0f}, zero = {0.0f, 0.0f, 0.0f};
    int32_t rc = FLUID_OK;
    for (int k = 0; k < frames && rc == FLUID_OK; ++k)
        rc = fluid_sim_frame(sim, gravity, zero, zero, 1.0f / 120.0f, 0, 16, (uint32_t)k);
    if (rc != FLUID_OK) return fail("fluid_sim_frame", rc);
    FluidSimStats st;
    rc = fluid_sim_stats(sim, &st);
    if (rc != FLUID_OK) return fail("fluid_sim_stats", rc);
    const uint32_t n = fluid_sim_count(sim);
    float *pos = (float *)malloc(16 * (size_t)n), *vel = (float *)malloc(16 * (size_t)n);
    if (!pos || !vel) return fail("malloc", -1);
    rc = fluid_sim_read_particles(sim, pos, vel);
    if (rc != FLUID_OK) return fail("fluid_sim_read_particles", rc);
    printf("n %u substeps %llu compression_avg %08x v_max %08x\n", (unsigned)n,
           (unsigned long long)st.substeps, (unsigned)bits(st.compression_avg),
           (unsigned)bits(st.v_max));
    if (argc > 2) {
        FILE *f = fopen(argv[2], "wb");
        if (!f || fwrite(pos, 16, n, f) != n || fwrite(vel, 16, n, f) != n || fclose(f) != 0)
            return fail("write particles", -1);
    }
    free(pos);
    free(vel);
    fluid_sim_destroy(sim);
    return 0;
}
