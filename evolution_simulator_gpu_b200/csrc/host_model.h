// Internal declarations shared by the host sources of the engine library.
#pragma once
#include <cstdint>
#include <string>

#include "../../include/creature_engine.h"

namespace ce {
extern thread_local std::string g_last_error;
void set_error(const std::string& msg);

uint32_t quake_hash(uint64_t id);
float quake_phase(uint32_t h);
float quake_scale(uint32_t h);
float terrain_amplitude(uint32_t level);
uint16_t f32_to_f16(float v);
float f16_to_f32(uint16_t h);
void ground(float x, float amplitude, float tilt, float width, float hurdle, float phase, float& h,
            float& s);

bool validate_body(const ce_population& pop, size_t i, std::string* why);
void fill_creature(const ce_population& pop, size_t i, const ce_world& w, uint32_t* record,
                   float* muscles, uint32_t* head, uint32_t record_at, uint32_t muscle_at);

uint32_t world_rate(const ce_world& w);
uint32_t world_settle(const ce_world& w);
uint32_t world_sample(const ce_world& w);
uint32_t world_steps(const ce_world& w);
float world_air_per_step(const ce_world& w);
// The mean heights where the niche's height bin steps up (metrics epilogue).
void height_bin_thresholds(float out[5]);

}  // namespace ce
