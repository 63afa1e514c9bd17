// Host camera math in float, in the reference's operation order.
#pragma once

#include <vector>

#include "rvsb.h"

namespace rvsb {

// Parameters::getRotationMatrix (Parameters.cpp:151-155):
// Rz(yaw) * Ry(pitch) * Rx(roll) of 0.01745329252f * rotation (degrees).
void rotation_matrix(const float rot_deg[3], float R[9]);

// SpaceTransformer::get_rotation / get_translation (SpaceTransformer.cpp:77-92).
void relative_pose(const rvsb_camera& in, const rvsb_camera& virt, float R[9], float t[3]);

// Equirectangular unprojection tables (EquirectangularUnprojector.cpp:55-98):
// rows: (cos theta_i, sin theta_i), columns: (cos phi_j, sin phi_j), with
// theta/phi evaluated in float and the trigonometric values rounded
// correctly to float.
void erp_tables(const rvsb_camera& in, std::vector<float>& rows, std::vector<float>& cols);

// Direction cones of an ERP input's vertex tiles (tile x tile pixels, each
// grown by one pixel on every side and clamped to the image), four floats
// per tile in row-major tile order: the unit direction of the region's
// middle pixel and an angle in radians bounding the angle from it to every
// pixel direction of the region (from the unprojection tables).
void erp_tile_cones(const rvsb_camera& in, const std::vector<float>& rows, const std::vector<float>& cols,
                    int tile, std::vector<float>& out);

// Projector constants of EquirectangularProjector.cpp:66-72.
void erp_projector_constants(const rvsb_camera& virt, float& u0, float& v0, float& du_dphi,
                             float& dv_dtheta);

// Validates a camera for synthesis; returns an error message or empty.
const char* camera_problem(const rvsb_camera& c, bool as_output);

}  // namespace rvsb
