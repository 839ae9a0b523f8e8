// Library-internal access to a frame handle for the request server (server.cu). Not part of the C ABI.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>

#include "../../include/depth_cuda.h"

namespace ds {

// The checks of ds_create (reference limits and the stages off the hot path); DS_OK or the error code.
int validate_params(const ds_stereo_params& params, int width, int height, std::string& message);

// A handle whose cost and path-value volumes belong to its owner: sized, never allocated, bound with
// bind_volumes before every frame. All other buffers are the handle's own; its census buffers have
// room for any min_disparity, so that set_frame_params never allocates.
int create_shared_volume_handle(const ds_stereo_params* params, int width, int height, ds_handle** out);
// Bytes of cost and path-value volume a frame of this handle needs (what bind_volumes must provide).
size_t volume_bytes(const ds_handle* h);
// `base` is device memory of volume_bytes(h) bytes, 256-byte aligned, unused by any frame in flight.
void bind_volumes(ds_handle* h, void* base);
// Remap tables owned by the caller (device f32 arrays lx, ly, rx, ry of map_w x map_h) used in place;
// the handle keeps its own raw-input buffers of raw_w x raw_h. Validation as ds_set_rectification.
int bind_rectification(ds_handle* h, float* const maps[4], int map_w, int map_h, int raw_w, int raw_h);
// Frame parameters that differ from the handle's only in min_disparity (the census guards follow it).
int set_frame_params(ds_handle* h, const ds_stereo_params& p);
// The handle's device buffers: inputs (raw when `raw`, else rectified; tightly packed) and outputs.
void input_buffers(ds_handle* h, bool raw, uint8_t* out[2]);
ds_outputs device_outputs(ds_handle* h);
int input_width(const ds_handle* h, bool raw);
int input_height(const ds_handle* h, bool raw);

}  // namespace ds
