// controller.cu — the per-frame controller around the step (host only).
//
// Restates the CPU side of Renderer::frame (crates/fluid-core/src/render.rs:
// 3021-3098): the body force from a motion sample (lib.rs:34-36), its
// adaptive smoothing (ForceFilter, render.rs:862-904), the gyroscope's
// smoothing and derivative (RotationTracker, :987-1016), the fingers on the
// glass (Fingers, :915-985), the idle gate that sleeps a settled pool
// (IdleGate, :1024-1105), the frame dt clamp (MAX_DT, :23) and the substep
// policy (substeps_for, :57-106). A frame's outcome is a FluidFramePlan; the
// GPU side runs it with fluid_sim_frame_plan.
#include <cmath>
#include <cstring>

#include "../../include/fluid_cu.h"

namespace {

constexpr float kStandardGravity = 9.80665f;  // lib.rs:5
constexpr float kMaxDt = 1.0f / 30.0f;        // render.rs:23
constexpr int kSlots = FLUID_TOUCH_SLOTS;

// render.rs:57-106, in f32 as the reference computes it.
constexpr float kSubstepPerSpacing = 0.42f;
constexpr float kRefineShortDt = 0.00105f;
constexpr float kNominalFrame = 1.0f / 120.0f;
constexpr float kCheapRungCost = 0.65f;

uint32_t sat_u32f(float v) {  // Rust's saturating `as u32`
    if (!(v > 0.0f)) return 0u;
    if (v >= 4294967296.0f) return 0xffffffffu;
    return (uint32_t)v;
}

float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }

struct ForceFilter {  // render.rs:862-904
    float smooth[3] = {0, 0, 0};
    bool started = false;
    float apply(const float force[3], float out[3]) {
        if (!started) {
            started = true;
            for (int i = 0; i < 3; ++i) smooth[i] = force[i];
        }
        float sum = 0.0f;
        for (int i = 0; i < 3; ++i) {
            const float d = force[i] - smooth[i];
            sum += d * d;
        }
        const float dev = std::sqrt(sum);
        const float alpha = clampf(dev / 2.0f, 0.02f, 1.0f);
        for (int i = 0; i < 3; ++i) smooth[i] += (force[i] - smooth[i]) * alpha;
        for (int i = 0; i < 3; ++i) out[i] = smooth[i];
        return dev;
    }
};

struct RotationTracker {  // render.rs:987-1016
    float smooth[3] = {0, 0, 0};
    bool primed = false;
    void apply(const float omega[3], float dt, float out[3], float domega[3]) {
        if (!primed || dt <= 0.0f || dt > 0.1f) {
            primed = true;
            for (int i = 0; i < 3; ++i) {
                smooth[i] = omega[i];
                out[i] = omega[i];
                domega[i] = 0.0f;
            }
            return;
        }
        const float alpha = 1.0f - std::exp(-dt / 0.025f);
        float prev[3];
        for (int i = 0; i < 3; ++i) prev[i] = smooth[i];
        for (int i = 0; i < 3; ++i) smooth[i] += (omega[i] - smooth[i]) * alpha;
        for (int i = 0; i < 3; ++i) {
            out[i] = smooth[i];
            domega[i] = clampf((smooth[i] - prev[i]) / dt, -200.0f, 200.0f);
        }
    }
};

struct Fingers {  // render.rs:915-985
    static constexpr float kRadius = 4.0f * 0.025f;  // WORLD_SCALE * 25 mm
    static constexpr float kSmoothTau = 0.02f;
    bool down[kSlots] = {};
    float at[kSlots][2] = {};
    float world[kSlots][2] = {};
    float velocity[kSlots][2] = {};
    bool tracked[kSlots] = {};
    bool any_down() const {
        for (int s = 0; s < kSlots; ++s)
            if (down[s]) return true;
        return false;
    }
    // Fills the Step block's finger tail: radius, count, packed live fingers.
    void step(const float extent[2], float dt, FluidStep &st) {
        st.touch_r = kRadius;
        st.touch_n = 0;
        for (int s = 0; s < kSlots; ++s) {
            if (!down[s]) {
                tracked[s] = false;
                continue;
            }
            const float x = at[s][0], y = at[s][1];
            const float w[2] = {(2.0f * x - 1.0f) * extent[0], (1.0f - 2.0f * y) * extent[1]};
            if (tracked[s] && dt > 0.0f) {
                const float alpha = 1.0f - std::exp(-dt / kSmoothTau);
                for (int a = 0; a < 2; ++a)
                    velocity[s][a] += ((w[a] - world[s][a]) / dt - velocity[s][a]) * alpha;
            } else {
                velocity[s][0] = velocity[s][1] = 0.0f;
            }
            world[s][0] = w[0];
            world[s][1] = w[1];
            tracked[s] = true;
            float *t = st.touches[st.touch_n];
            t[0] = w[0];
            t[1] = w[1];
            t[2] = velocity[s][0];
            t[3] = velocity[s][1];
            st.touch_n++;
        }
    }
};

struct IdleGate {  // render.rs:1024-1105
    static constexpr float kVSleep = 0.04f;
    static constexpr float kDevSleep = 0.5f;
    static constexpr uint32_t kStillFrames = 180;
    static constexpr float kDevWake = 1.2f;
    static constexpr float kCosWake = 0.999657f;
    static constexpr float kMagWake = 0.3f;
    static constexpr float kOmegaWake = 0.05f;
    uint32_t still = 0;
    bool sleeping = false;
    float sleep_force[3] = {0, 0, 0};
    static float dot(const float a[3], const float b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
    bool asleep(bool touched, const float smooth[3], float dev, const float omega[3], float v_max) {
        if (touched) {
            sleeping = false;
            still = 0;
            return false;
        }
        const bool spinning = std::sqrt(dot(omega, omega)) > kOmegaWake;
        if (sleeping) {
            const float m = std::sqrt(dot(smooth, smooth) * dot(sleep_force, sleep_force));
            const float cos = dot(smooth, sleep_force) / (m > 1e-6f ? m : 1e-6f);
            const float mag_shift = std::fabs(std::sqrt(dot(smooth, smooth)) - std::sqrt(dot(sleep_force, sleep_force)));
            if (dev > kDevWake || cos < kCosWake || mag_shift > kMagWake || spinning) {
                sleeping = false;
                still = 0;
                return false;
            }
            return true;
        }
        if (v_max < kVSleep && dev < kDevSleep && !spinning) {
            still += 1;
            if (still >= kStillFrames) {
                sleeping = true;
                for (int i = 0; i < 3; ++i) sleep_force[i] = smooth[i];
                return true;
            }
        } else {
            still = 0;
        }
        return false;
    }
};

}  // namespace

struct FluidController {
    float spacing = 0.0f;
    float extent[2] = {0, 0};
    uint32_t cap = 16;
    uint64_t frames = 0;
    uint64_t idle_frames = 0;
    double last_frame_ms = 0.0;
    uint32_t frame_seed = 0;
    ForceFilter force;
    RotationTracker rotation;
    Fingers fingers;
    IdleGate idle;
};

extern "C" {

uint32_t fluid_substep_floor(float dt, float dt_sub_max) {  // render.rs:63-65
    const uint32_t n = sat_u32f(std::ceil(dt / dt_sub_max));
    return n < 8u ? n : 8u;
}

uint32_t fluid_refine_passes(float dt_sub) { return dt_sub > kRefineShortDt ? 5u : 2u; }  // :76-78

float fluid_field_keep_target(float v_max) {  // render.rs:1107-1111, FIELD_KEEP :517
    float t = (v_max - 0.05f) / 0.20f;
    t = t < 0.0f ? 0.0f : (t > 1.0f ? 1.0f : t);
    return 0.8f * (1.0f - t * t * (3.0f - 2.0f * t));
}

uint32_t fluid_substeps_for(float dt, float v_max, float spacing, uint32_t cap) {  // :97-106
    uint32_t n = sat_u32f(std::ceil(dt * v_max / (0.4f * spacing)));
    const uint32_t fl = fluid_substep_floor(dt, kSubstepPerSpacing * spacing);
    if (fl > n) n = fl;
    const uint32_t cheap = sat_u32f(std::ceil(kNominalFrame / kRefineShortDt));
    const bool jump = fluid_refine_passes(dt / (float)cheap) == 2u && n < cheap &&
                      (float)n > kCheapRungCost * (float)cheap;
    if (jump) n = cheap;
    return n < cap ? n : cap;
}

struct FluidIdleGate {
    IdleGate g;
};

FluidIdleGate *fluid_idle_gate_create(void) { return new FluidIdleGate(); }
void fluid_idle_gate_destroy(FluidIdleGate *g) { delete g; }
uint32_t fluid_idle_gate_still_frames(void) { return IdleGate::kStillFrames; }
uint32_t fluid_idle_gate_asleep(FluidIdleGate *g, uint32_t touched, const float smooth[3], float dev,
                                const float omega[3], float v_max) {
    if (!g || !smooth || !omega) return 0u;
    return g->g.asleep(touched != 0, smooth, dev, omega, v_max) ? 1u : 0u;
}

FluidController *fluid_controller_create(float spacing, const float extent[2], uint32_t cap) {
    if (!(spacing > 0.0f) || !extent || !(extent[0] > 0.0f) || !(extent[1] > 0.0f)) return nullptr;
    FluidController *c = new FluidController();
    c->spacing = spacing;
    c->extent[0] = extent[0];
    c->extent[1] = extent[1];
    c->cap = cap ? cap : 16u;
    return c;
}

void fluid_controller_destroy(FluidController *c) { delete c; }

int32_t fluid_controller_touch(FluidController *c, uint32_t slot, float x, float y, uint32_t down) {
    if (!c) return FLUID_ERR_ARG;
    if (slot >= (uint32_t)kSlots) return FLUID_OK;  // render.rs:2986-2990 ignores unknown slots
    c->fingers.down[slot] = down != 0;
    c->fingers.at[slot][0] = x;
    c->fingers.at[slot][1] = y;
    return FLUID_OK;
}

int32_t fluid_controller_plan(FluidController *c, const FluidMotion *m, double now_ms, float v_max,
                              FluidFramePlan *out) {
    if (!c || !m || !out) return FLUID_ERR_ARG;
    std::memset(out, 0, sizeof *out);
    const float interval_us = (float)((now_ms - c->last_frame_ms) * 1000.0);
    const float body[3] = {kStandardGravity * (m->gravity.x + m->user_acceleration.x),
                           kStandardGravity * (m->gravity.y + m->user_acceleration.y),
                           kStandardGravity * (m->gravity.z + m->user_acceleration.z)};
    float force[3], omega[3], domega[3];
    const float dev = c->force.apply(body, force);
    const float rot[3] = {m->rotation_rate.x, m->rotation_rate.y, m->rotation_rate.z};
    c->rotation.apply(rot, interval_us / 1000000.0f, omega, domega);
    out->force = FluidVec3{force[0], force[1], force[2]};
    out->omega = FluidVec3{omega[0], omega[1], omega[2]};
    out->domega = FluidVec3{domega[0], domega[1], domega[2]};
    out->deviation = dev;
    if (c->idle.asleep(c->fingers.any_down(), force, dev, omega, v_max)) {
        c->last_frame_ms = now_ms;
        c->idle_frames += 1;
        out->asleep = 1;
        return FLUID_OK;
    }
    c->last_frame_ms = now_ms;
    const float dt = c->frames == 0 ? 0.0f : clampf(interval_us / 1000000.0f, 0.0f, kMaxDt);
    out->dt = dt;
    FluidStep &st = out->step;
    c->fingers.step(c->extent, dt, st);
    out->substeps = dt > 0.0f ? fluid_substeps_for(dt, v_max, c->spacing, c->cap) : 0u;
    c->frame_seed += 1u;
    out->seed = c->frame_seed;
    if (out->substeps) {
        const float dt_sub = dt / (float)out->substeps;
        st.force[0] = force[0];
        st.force[1] = force[1];
        st.force[2] = force[2];
        st.dt = dt_sub;
        st.omega[0] = omega[0];
        st.omega[1] = omega[1];
        st.omega[2] = omega[2];
        st.v_clamp = 0.4f * c->spacing / dt_sub;  // render.rs:3171
        st.domega[0] = domega[0];
        st.domega[1] = domega[1];
        st.domega[2] = domega[2];
        st.seed = 0;
        out->refine = fluid_refine_passes(dt_sub);
    }
    c->frames += 1;
    out->frames = c->frames;
    out->idle_frames = c->idle_frames;
    return FLUID_OK;
}

}  // extern "C"
