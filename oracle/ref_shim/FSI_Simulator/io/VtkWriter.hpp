// Stand-in for the reference's include/FSI_Simulator/io/VtkWriter.hpp when
// its fluid-step sources are compiled into oracle/_ref: the writer needs VTK
// (not installed here) and only LbmFlowField2D/3D::saveFrameData calls it,
// which the checker never does.
#pragma once

namespace fsi {
namespace io {
struct VtkWriter {
    template <typename... A> static void writeImageDataVectorField(A &&...) {}
    template <typename... A> static void writeImageDataScalarField(A &&...) {}
};
} // namespace io
} // namespace fsi
