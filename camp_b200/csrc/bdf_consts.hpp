// Constants of the CVODE BDF method and of CAMP's state handling, shared by
// the two device kernels (warp-per-cell and lane-per-cell).
#pragma once

namespace campb {
namespace bdf {

constexpr double kSmall = 1.0e-30;  // src/camp_common.h:44
constexpr double kTiny = 1.0e-60;   // src/camp_common.h:45

// CVODE constants (Hindmarsh et al., ACM TOMS 31(3) 2005; CVODE documentation)
constexpr int QMAX = 5;
constexpr int LMAX = QMAX + 1;
constexpr double ETAMX1 = 10000.0, ETAMX2 = 10.0, ETAMX3 = 10.0;
constexpr double ETAMXF = 0.2, ETAMIN = 0.1, ETACF = 0.25;
constexpr double ADDON = 0.000001, BIAS1 = 6.0, BIAS2 = 6.0, BIAS3 = 10.0;
constexpr double THRESH = 1.5;
constexpr int SMALL_NST = 10, MXNEF1 = 3, SMALL_NEF = 2, LONG_WAIT = 10;
constexpr int MAXCOR = 3;
constexpr double CRDOWN = 0.3, DGMAX = 0.3, RDIV = 2.0;
constexpr int MSBP = 20, MSBJ = 50;
constexpr double DGMAX_J = 0.2, NLSCOEF = 0.1;
constexpr double UROUND = 2.220446049250313e-16;

// outcome codes (CVODE flags)
constexpr int OK = 0, TOO_MUCH_WORK = -1, TOO_MUCH_ACC = -2, ERR_FAILURE = -3,
              CONV_FAILURE = -4, REPTD_RHSFUNC_ERR = -10, UNREC_RHSFUNC_ERR = -11,
              ILL_INPUT = -22, TOO_CLOSE = -27;
// nonlinear solver outcomes
constexpr int NL_OK = 0, NL_CONV_FAIL = 1, NL_RHS_RECVR = 2, NL_TRY_AGAIN = 3,
              NL_CONSTR_RECVR = 4;
constexpr int NO_FAILURES = 0, FAIL_BAD_J = 1, FAIL_OTHER = 2;
constexpr int FIRST_CALL = 0, PREV_CONV_FAIL = 1, PREV_ERR_FAIL = 2;

}  // namespace bdf
}  // namespace campb
