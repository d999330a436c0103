// rkf78.h -- Fehlberg's 7(8) Runge-Kutta pair (E. Fehlberg, NASA TR R-287,
// 1968), the method of boost::odeint's runge_kutta_fehlberg78 that the
// reference steps with (src/tdse/tdse.cpp:171,190).  Coefficients are the
// doubles nearest the published fractions.
#pragma once

namespace rkf78 {

#define F_(p, q) (double(p) / double(q))
constexpr double C[13] = {0, F_(2, 27), F_(1, 9), F_(1, 6), F_(5, 12), F_(1, 2), F_(5, 6),
                          F_(1, 6), F_(2, 3), F_(1, 3), 1, 0, 1};

constexpr double A[13][13] = {
    {0},
    {F_(2, 27)},
    {F_(1, 36), F_(1, 12)},
    {F_(1, 24), 0, F_(1, 8)},
    {F_(5, 12), 0, F_(-25, 16), F_(25, 16)},
    {F_(1, 20), 0, 0, F_(1, 4), F_(1, 5)},
    {F_(-25, 108), 0, 0, F_(125, 108), F_(-65, 27), F_(125, 54)},
    {F_(31, 300), 0, 0, 0, F_(61, 225), F_(-2, 9), F_(13, 900)},
    {2, 0, 0, F_(-53, 6), F_(704, 45), F_(-107, 9), F_(67, 90), 3},
    {F_(-91, 108), 0, 0, F_(23, 108), F_(-976, 135), F_(311, 54), F_(-19, 60), F_(17, 6),
     F_(-1, 12)},
    {F_(2383, 4100), 0, 0, F_(-341, 164), F_(4496, 1025), F_(-301, 82), F_(2133, 4100),
     F_(45, 82), F_(45, 164), F_(18, 41)},
    {F_(3, 205), 0, 0, 0, 0, F_(-6, 41), F_(-3, 205), F_(-3, 41), F_(3, 41), F_(6, 41), 0},
    {F_(-1777, 4100), 0, 0, F_(-341, 164), F_(4496, 1025), F_(-289, 82), F_(2193, 4100),
     F_(51, 82), F_(33, 164), F_(12, 41), 0, 1},
};

// 8th-order weights: the propagated solution.
constexpr double B8[13] = {0, 0, 0, 0, 0, F_(34, 105), F_(9, 35), F_(9, 35), F_(9, 280),
                           F_(9, 280), 0, F_(41, 840), F_(41, 840)};
// 7th-order weights: used only through the embedded error estimate.
constexpr double B7[13] = {F_(41, 840), 0, 0, 0, 0, F_(34, 105), F_(9, 35), F_(9, 35),
                           F_(9, 280), F_(9, 280), F_(41, 840), 0, 0};
// Coefficients of the 8th-order solution's stability polynomial
// R(z) = 1 + z b8^T (I - zA)^{-1} 1 = sum_m G[m] z^m: G[m] = b8^T A^(m-1) 1
// for m >= 1, evaluated in exact rational arithmetic from the fractions
// above.  G[m] = 1/m! up to m = 8 (the method's order); the z^13 coefficient
// vanishes (a_{11,10} = 0 breaks the only chain through all 13 stages), so
// R has degree 12.  With the field frozen over a step the system is linear
// and autonomous, and one step is x_new = R(hM) x exactly (up to rounding).
constexpr double G[13] = {1,
                          1,
                          F_(1, 2),
                          F_(1, 6),
                          F_(1, 24),
                          F_(1, 120),
                          F_(1, 720),
                          F_(1, 5040),
                          F_(1, 40320),
                          F_(491, 209018880),
                          F_(1333, 5643509760LL),
                          F_(-13, 501645312),
                          F_(-65, 4514807808LL)};
#undef F_

}  // namespace rkf78

// |R(iy)| <= 1 for 0 <= y <= this bound, R the stability polynomial of the
// 8th-order solution (computed from the tableau above).
constexpr double kRk78ImagStability = 2.365;
