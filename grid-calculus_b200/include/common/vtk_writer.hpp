// Drop-in for the reference's examples/common/vtk_writer.hpp: the legacy
// ASCII VTK STRUCTURED_POINTS writer, written by the library
// (gc_write_vtk) with the reference's bytes.  Device-resident fields are
// snapshotted without stalling the computation through gc_snapshotter
// (gridcalc_b200.h).
#pragma once

#include <stdexcept>
#include <string>

#include <gridcalc/b200.hpp>

namespace gridcalc::examples {

// writeVtkStructuredPoints (examples/common/vtk_writer.hpp:34-66); throws
// std::runtime_error when the file cannot be written, as the reference does.
inline void writeVtkStructuredPoints(const core::Field<double>& field, const std::string& path,
                                     const std::string& field_name) {
  const gc_grid g = field.getGrid().c();
  if (gc_write_vtk(&g, GC_F64, field.data(), path.c_str(), field_name.c_str(), GC_VTK_ASCII) != GC_OK)
    throw std::runtime_error(gc_last_error());
}

}  // namespace gridcalc::examples
