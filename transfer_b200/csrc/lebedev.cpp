// LebedevQuad (see angular.h).
#include <stdexcept>

#include "angular.h"

namespace transfer {

// Orders and algebraic precisions of the Lebedev-Laikov family
// (order_by_precision, LebedevQuad.cpp:8-30).
static const int kOrders[] = {6,    14,   26,   38,   50,   74,   86,   110,  146,  170,  194,  230,  266,
                              302,  350,  386,  434,  482,  530,  590,  650,  698,  770,  830,  890,  974,
                              1046, 1118, 1202, 1274, 1358, 1454, 1538, 1622, 1730, 1814, 1910, 2030, 2126,
                              2222, 2354, 2450, 2558, 2702, 2810, 2930, 3074, 3182, 3314, 3470, 3590, 3722,
                              3890, 4010, 4154, 4334, 4466, 4610, 4802, 4934, 5090, 5294, 5438, 5606, 5810};

int lebedev_order_by_precision(int prec) {
    for (int i = 0; i < 65; ++i)
        if (3 + 2 * i >= prec) return kOrders[i];
    return -1;
}

LebedevQuad::LebedevQuad(int mindegree) {
    order = lebedev_order_by_precision(mindegree);
    throw std::runtime_error("LebedevQuad: rule generation not available in this build");
}

}  // namespace transfer
