// Internal interface between the mortar space (mortar.cu) and the AMR step (amr.cu): the AMR
// stage kernel adds the mortar lifts itself, in the order the lift kernel would, so the step
// needs the face kernel alone and the device lists the lift kernel reads.
#pragma once
#include <cstdint>

struct drf_mortar;

namespace drf {

struct MortarLifts {
    const double *contrib;  // [interface][slot][face node] staged lifts
    const int64_t *touched; // elements touched by an interface
    const int64_t *ptr;     // entries of touched element u: ent[ptr[u] .. ptr[u + 1])
    const int *ent;         // (interface, slot, face) triples
    int64_t n_touched;
    int slots;              // slots per interface (coarse side + fine faces)
};

// Enqueues the mortar face kernel on the handle's stream: every interface's lifts of the
// scalar field d_U (device) staged for MortarLifts::contrib.
void mortar_stage_faces(drf_mortar *h, int kind, const double a[3], const double *d_U);
MortarLifts mortar_lifts(const drf_mortar *h);

}  // namespace drf
