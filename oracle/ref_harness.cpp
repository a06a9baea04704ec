// Host-side harness around the reference's own RRSWeightWindow
// (src/render/common/commoncudautils.h:14-28), compiled from the reference checkout by
// oracle/Makefile into oracle/_ref/. Test infrastructure: it pins oracle_weight_window_f32.
#include "render/common/commoncudautils.h"

extern "C" float ref_rrs_weight_window(float x, float ww) { return RRSWeightWindow(x, ww); }
