// tight_inclusion/ccd.hpp — TEST-ONLY stand-in for the Tight-Inclusion CCD
// header that tools/scene_object_envelope_native_ti_walltime.cpp includes.
//
// Tight-Inclusion (ticcd) is a third-party dependency that the reference does
// not vendor.  This header declares only the names that tool uses
// (Scalar, Vector3, Array3, CCDRootFindingMethod, vertexFaceCCD, edgeEdgeCCD)
// so the tool compiles unchanged; oracle/ref_tool.cpp defines the two queries
// by forwarding to the reference's own certifier
// (EvaluatePointTriangleInterval / EvaluateEdgeEdgeInterval,
// cpp/certificate/certificate_engine.cpp:481-551) and reporting a hit for
// collision or undecided, the conservative decision mapping.  Never part of
// the product.
#pragma once

namespace ticcd {

using Scalar = double;

struct Vector3 {
  double v[3];
  Vector3(double x, double y, double z) : v{x, y, z} {}
  double operator[](int i) const { return v[i]; }
};

struct Array3 {
  double v[3];
  Array3(double x, double y, double z) : v{x, y, z} {}
};

enum class CCDRootFindingMethod { DEPTH_FIRST_SEARCH, BREADTH_FIRST_SEARCH };

bool vertexFaceCCD(const Vector3& vertex_start, const Vector3& face_vertex0_start,
                   const Vector3& face_vertex1_start, const Vector3& face_vertex2_start,
                   const Vector3& vertex_end, const Vector3& face_vertex0_end,
                   const Vector3& face_vertex1_end, const Vector3& face_vertex2_end,
                   const Array3& err, Scalar ms, Scalar& toi, Scalar tolerance, Scalar t_max,
                   long max_itr, Scalar& output_tolerance, bool no_zero_toi,
                   CCDRootFindingMethod method);

bool edgeEdgeCCD(const Vector3& edge0_vertex0_start, const Vector3& edge0_vertex1_start,
                 const Vector3& edge1_vertex0_start, const Vector3& edge1_vertex1_start,
                 const Vector3& edge0_vertex0_end, const Vector3& edge0_vertex1_end,
                 const Vector3& edge1_vertex0_end, const Vector3& edge1_vertex1_end,
                 const Array3& err, Scalar ms, Scalar& toi, Scalar tolerance, Scalar t_max,
                 long max_itr, Scalar& output_tolerance, bool no_zero_toi,
                 CCDRootFindingMethod method);

}  // namespace ticcd
