// ns3d_shim.h -- what a host that links the Field3D shim (ns3d_shim.cpp) adds
// beyond the reference's own entry points.
//
// The shim keeps the state on the GPU between calls. Field3D's arrays are
// brought up to date by the shim's output functions (write_tecplot_field) and
// by ns3d_shim_sync; the device takes Field3D's arrays again after
// ns3d_shim_invalidate. The reference's time_advance and main need neither.
#pragma once

#include "field_structures.h"

// Copy the device state into F (rho..E, u,v,w,p,T,c, ghost faces included)
// when the device holds a newer state than F's arrays; a no-op otherwise.
void ns3d_shim_sync(Field3D& F);

// F's arrays were changed on the host: the next shimmed call uploads them.
void ns3d_shim_invalidate(const Field3D& F);
