// wigtable.cpp — the registry of WigTable kick tables (AWigTable, reference accel.h:403-425).
//
// The reference keeps each table inside its element object (xl[MAX_WIGTAB_X], yl, xkick[my][mx],
// ykick[my][mx]).  Descriptors here are plain fixed-size records, so a table lives in this
// process-wide registry and an element names it by id (accel_elem_desc.f[0]).  Tables are
// immutable once created; a line copies the ones it uses to its device when it is compiled.
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include "engine.h"

namespace accel {

namespace {
std::mutex g_mu;
std::map<int32_t, std::shared_ptr<const WigTab>> g_tabs;
int32_t g_next = 1;

bool monotonic(const double* v, int n) {
    bool up = v[n - 1] > v[0];
    for (int i = 0; i + 1 < n; i++) {
        if (!(std::isfinite(v[i]) && std::isfinite(v[i + 1]))) return false;
        if (up ? !(v[i + 1] > v[i]) : !(v[i + 1] < v[i])) return false;
    }
    return true;
}
}  // namespace

std::shared_ptr<const WigTab> wigtable_find(int32_t id) {
    std::lock_guard<std::mutex> g(g_mu);
    auto it = g_tabs.find(id);
    return it == g_tabs.end() ? nullptr : it->second;
}

int wigtable_register(int mx, int my, const double* xl, const double* yl, const double* xkick,
                      const double* ykick, int32_t* id, std::string& err) {
    if (mx < 2 || mx > kWigTabMaxX || my < 2 || my > kWigTabMaxY) {
        err = "WigTable size " + std::to_string(mx) + " x " + std::to_string(my) +
              " outside 2..101 x 2..21";
        return ACCEL_E_INVALID;
    }
    if (!monotonic(xl, mx) || !monotonic(yl, my)) {
        err = "WigTable grid is not strictly monotonic";
        return ACCEL_E_INVALID;
    }
    auto t = std::make_shared<WigTab>();
    t->mx = mx;
    t->my = my;
    t->data.resize(wigtable_doubles(mx, my));
    double* p = t->data.data();
    std::memcpy(p, xl, sizeof(double) * mx);
    std::memcpy(p + mx, yl, sizeof(double) * my);
    std::memcpy(p + mx + my, xkick, sizeof(double) * mx * my);
    std::memcpy(p + mx + my + mx * my, ykick, sizeof(double) * mx * my);
    std::lock_guard<std::mutex> g(g_mu);
    *id = g_next++;
    g_tabs[*id] = std::move(t);
    return ACCEL_OK;
}

}  // namespace accel

using namespace accel;

extern "C" int accel_wigtable_create(int mx, int my, const double* xl, const double* yl,
                                     const double* xkick, const double* ykick, int32_t* id) {
    if (!xl || !yl || !xkick || !ykick || !id) return fail(ACCEL_E_INVALID, "NULL argument");
    std::string err;
    int s = wigtable_register(mx, my, xl, yl, xkick, ykick, id, err);
    return s ? fail(s, err) : ACCEL_OK;
}

extern "C" int accel_wigtable_info(int32_t id, int* mx, int* my) {
    auto t = wigtable_find(id);
    if (!t) return fail(ACCEL_E_INVALID, "no WigTable table with id " + std::to_string(id));
    if (mx) *mx = t->mx;
    if (my) *my = t->my;
    return ACCEL_OK;
}

extern "C" int accel_wigtable_get(int32_t id, double* xl, double* yl, double* xkick, double* ykick) {
    auto t = wigtable_find(id);
    if (!t) return fail(ACCEL_E_INVALID, "no WigTable table with id " + std::to_string(id));
    const int mx = t->mx, my = t->my;
    const double* p = t->data.data();
    if (xl) std::memcpy(xl, p, sizeof(double) * mx);
    if (yl) std::memcpy(yl, p + mx, sizeof(double) * my);
    if (xkick) std::memcpy(xkick, p + mx + my, sizeof(double) * mx * my);
    if (ykick) std::memcpy(ykick, p + mx + my + mx * my, sizeof(double) * mx * my);
    return ACCEL_OK;
}

extern "C" int accel_wigtable_destroy(int32_t id) {
    std::lock_guard<std::mutex> g(g_mu);
    if (!g_tabs.erase(id)) return fail(ACCEL_E_INVALID, "no WigTable table with id " + std::to_string(id));
    return ACCEL_OK;
}
