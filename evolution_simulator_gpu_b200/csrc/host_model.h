// Internal declarations shared by the host sources of the engine library.
#pragma once
#include <cstdint>
#include <string>

#include "../../include/creature_engine.h"

namespace ce {
extern thread_local std::string g_last_error;
void set_error(const std::string& msg);

float f16_to_f32(uint16_t h);
// The quake hash, terrain amplitude, f32 -> f16 rounding and ground of the
// packer are in packer.h, shared with the device packer.

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
