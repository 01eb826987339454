// fields.cpp — element field access by id and the line-wide flag switches.
//
// Field names and rules follow the reference's setfield/getfield methods:
//   Length (all), K (Quad accel.cpp:216, Bend 498), PolynomB/PolynomA[index] (StrMPole
//   accel.cpp:773-785: index may equal MaxNPole; BendMPole 622-634: index < MaxNPole), NSlice,
//   MaxNPole, BendingAngle (refreshes irho = theta/len, accel.cpp:497,581), EntranceAngle,
//   ExitAngle, Voltage/Frequency/Phis/Energy (Cavity 870-885), KickX/KickY (Corrector 245-256),
//   XLim/YLim (Aperture 308-321).
// Flag switches follow ALine::set_rad_onoff / set_cavity_onoff / set_wake_onoff
// (aline.cpp:258-293, 429-463).
#include <cmath>
#include "engine.h"
#include "runtime.h"

namespace accel {

static int bad(const accel_elem_desc& d, int field) {
    return fail(ACCEL_E_INVALID, std::string("field ") + std::to_string(field) +
                                     " not present in element type " + type_name(d.type));
}

int desc_set_field(accel_elem_desc& d, int field, int index, const double* v) {
    const int t = d.type;
    switch (field) {
    case ACCEL_F_LENGTH: d.len = v[0]; return ACCEL_OK;
    case ACCEL_F_K:
        if (t == ACCEL_QUAD) { d.f[0] = v[0]; return ACCEL_OK; }
        if (t == ACCEL_BEND) { d.f[3] = v[0]; return ACCEL_OK; }
        if (t == ACCEL_STRMPOLE) { d.poly_b[1] = v[0]; return ACCEL_OK; }
        return bad(d, field);
    case ACCEL_F_POLYNOMB:
    case ACCEL_F_POLYNOMA: {
        const bool a = field == ACCEL_F_POLYNOMA;
        if (index < 0 || index >= ACCEL_MAX_MPOLE) return fail(ACCEL_E_INVALID, "multipole index outside 0..9");
        if (t == ACCEL_STRMPOLE) {
            if (index > d.max_npole) return fail(ACCEL_E_INVALID, "index > MaxNPole");
            (a ? d.poly_a : d.poly_b)[index] = v[0];
            return ACCEL_OK;
        }
        if (t == ACCEL_BENDMPOLE && !a) {
            if (index >= d.max_npole) return fail(ACCEL_E_INVALID, "index >= MaxNPole");
            d.poly_b[index] = v[0];
            return ACCEL_OK;
        }
        return bad(d, field);
    }
    case ACCEL_F_NSLICE:
        if (t == ACCEL_STRMPOLE || t == ACCEL_BENDMPOLE || t == ACCEL_IDEALWIG || t == ACCEL_WIGTABLE) {
            if (v[0] < 1) return fail(ACCEL_E_INVALID, "NSlice must be >= 1");
            d.nslice = (int)v[0];
            return ACCEL_OK;
        }
        return bad(d, field);
    case ACCEL_F_MAXNPOLE:
        if (t == ACCEL_STRMPOLE || t == ACCEL_BENDMPOLE || t == ACCEL_RFMULT) {
            if (v[0] < 0 || v[0] > ACCEL_MAX_MPOLE) return fail(ACCEL_E_INVALID, "MaxNPole outside 0..10");
            d.max_npole = (int)v[0];
            return ACCEL_OK;
        }
        return bad(d, field);
    case ACCEL_F_ANGLE:
        if (t == ACCEL_BEND || t == ACCEL_BENDMPOLE) { d.f[0] = v[0]; d.f[4] = d.f[0] / d.len; return ACCEL_OK; }
        return bad(d, field);
    case ACCEL_F_E1:
        if (t == ACCEL_BEND || t == ACCEL_BENDMPOLE) { d.f[1] = v[0]; return ACCEL_OK; }
        return bad(d, field);
    case ACCEL_F_E2:
        if (t == ACCEL_BEND || t == ACCEL_BENDMPOLE) { d.f[2] = v[0]; return ACCEL_OK; }
        return bad(d, field);
    case ACCEL_F_VOLTAGE:
        if (t == ACCEL_CAVITY) { d.f[0] = v[0]; return ACCEL_OK; }
        return bad(d, field);
    case ACCEL_F_FREQUENCY:
        if (t == ACCEL_CAVITY) { d.f[1] = v[0]; return ACCEL_OK; }
        return bad(d, field);
    case ACCEL_F_PHIS:
        if (t == ACCEL_CAVITY) { d.f[2] = v[0]; return ACCEL_OK; }
        return bad(d, field);
    case ACCEL_F_ENERGY:
        if (t == ACCEL_CAVITY || t == ACCEL_BENDMPOLE) { d.f[3] = v[0]; return ACCEL_OK; }
        if (t == ACCEL_TRANSWAKE || t == ACCEL_SYNCRAD || t == ACCEL_LONGWAKE) { d.f[0] = v[0]; return ACCEL_OK; }
        return bad(d, field);
    case ACCEL_F_KICKX:
        if (t == ACCEL_CORRECTOR) { d.f[0] = v[0]; return ACCEL_OK; }
        return bad(d, field);
    case ACCEL_F_KICKY:
        if (t == ACCEL_CORRECTOR) { d.f[1] = v[0]; return ACCEL_OK; }
        return bad(d, field);
    case ACCEL_F_XLIM:
        if (t == ACCEL_APERTURE) { d.f[0] = v[0]; d.f[1] = v[1]; return ACCEL_OK; }
        return bad(d, field);
    case ACCEL_F_YLIM:
        if (t == ACCEL_APERTURE) { d.f[2] = v[0]; d.f[3] = v[1]; return ACCEL_OK; }
        return bad(d, field);
    default:
        return fail(ACCEL_E_INVALID, "unknown field id");
    }
}

int desc_get_field(const accel_elem_desc& d, int field, int index, double* v) {
    accel_elem_desc tmp = d;
    const int t = d.type;
    switch (field) {
    case ACCEL_F_LENGTH: v[0] = d.len; return ACCEL_OK;
    case ACCEL_F_K:
        if (t == ACCEL_QUAD) { v[0] = d.f[0]; return ACCEL_OK; }
        if (t == ACCEL_BEND) { v[0] = d.f[3]; return ACCEL_OK; }
        if (t == ACCEL_STRMPOLE) { v[0] = d.poly_b[1]; return ACCEL_OK; }
        return bad(tmp, field);
    case ACCEL_F_POLYNOMB:
    case ACCEL_F_POLYNOMA:
        if (index < 0 || index >= ACCEL_MAX_MPOLE) return fail(ACCEL_E_INVALID, "multipole index outside 0..9");
        if (t == ACCEL_STRMPOLE) { v[0] = (field == ACCEL_F_POLYNOMA ? d.poly_a : d.poly_b)[index]; return ACCEL_OK; }
        if (t == ACCEL_BENDMPOLE && field == ACCEL_F_POLYNOMB) { v[0] = d.poly_b[index]; return ACCEL_OK; }
        return bad(tmp, field);
    case ACCEL_F_NSLICE: v[0] = d.nslice; return ACCEL_OK;
    case ACCEL_F_MAXNPOLE: v[0] = d.max_npole; return ACCEL_OK;
    case ACCEL_F_ANGLE: v[0] = d.f[0]; return ACCEL_OK;
    case ACCEL_F_E1: v[0] = d.f[1]; return ACCEL_OK;
    case ACCEL_F_E2: v[0] = d.f[2]; return ACCEL_OK;
    case ACCEL_F_VOLTAGE: v[0] = d.f[0]; return ACCEL_OK;
    case ACCEL_F_FREQUENCY: v[0] = d.f[1]; return ACCEL_OK;
    case ACCEL_F_PHIS: v[0] = d.f[2]; return ACCEL_OK;
    case ACCEL_F_ENERGY:
        v[0] = (t == ACCEL_CAVITY || t == ACCEL_BENDMPOLE) ? d.f[3] : d.f[0];
        return ACCEL_OK;
    case ACCEL_F_KICKX: v[0] = d.f[0]; return ACCEL_OK;
    case ACCEL_F_KICKY: v[0] = d.f[1]; return ACCEL_OK;
    case ACCEL_F_XLIM: v[0] = d.f[0]; v[1] = d.f[1]; return ACCEL_OK;
    case ACCEL_F_YLIM: v[0] = d.f[2]; v[1] = d.f[3]; return ACCEL_OK;
    default: return fail(ACCEL_E_INVALID, "unknown field id");
    }
}

// rad_flag / cavity_on / wake_on: a negative value leaves that switch unchanged.
void apply_flags(accel_elem_desc* d, int n, int rad_flag, int cavity_on, int wake_on) {
    for (int k = 0; k < n; k++) {
        accel_elem_desc& e = d[k];
        if (rad_flag >= 0) {
            if (e.type == ACCEL_BENDMPOLE || e.type == ACCEL_IDEALWIG)
                e.flags = (rad_flag <= 2) ? rad_flag : 0;
            else if (e.type == ACCEL_SYNCRAD)
                e.flags = rad_flag == ACCEL_RAD_LUMP ? 3 : rad_flag == ACCEL_RAD_LUMP_DAMP ? 1
                        : rad_flag == ACCEL_RAD_LUMP_QE ? 2 : 0;
        }
        if (cavity_on >= 0 && e.type == ACCEL_CAVITY) e.flags = cavity_on ? 1 : 0;
        if (wake_on >= 0 && (e.type == ACCEL_TRANSWAKE || e.type == ACCEL_LONGWAKE)) e.flags = wake_on ? 1 : 0;
    }
}

}  // namespace accel
