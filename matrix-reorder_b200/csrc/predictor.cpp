// Ridge "headroom" predictor over the 10 reuse-distance bin probabilities.
//
// The model is log(speedup) = b + sum_i w_i r_i with the raw (scaler-folded)
// coefficients the reference's trainer exported; the numbers below are the
// reference's published model tables (data, kept as published):
//   MERBIT sampled: include/model.cuh:81-95 (= ridge/out/merbit/sampled/rd_sampled_merbit_model.hpp)
//   MERBIT exact:   ridge/out/merbit/exact/rd_exact_merbit_model.hpp
//   CSR sampled:    ridge/out/csr/sampled/rd_sampled_csr_model.hpp
//   CSR exact:      ridge/out/csr/exact/rd_exact_csr_model.hpp
// Evaluation order (intercept first, then features 0..9) follows
// PredictLogSpeedup (include/model.cuh:84-89) so results match bit for bit.
#include <cmath>

#include "mr.h"

namespace {

struct RidgeModel {
    double coef[10];
    double intercept;
};

const RidgeModel kModels[4] = {
    {{-3.36257371695098284e-01, -2.55786219126070413e-01, -2.42480790872360380e-01, -6.03012191232085021e-02,
      2.80536873107643969e-01, -1.63999842129305441e-02, -4.63437995705341804e-02, -3.01657913615571149e-01,
      2.75407122122610781e+00, 2.30428797617423475e+00},
     2.66499564016047963e-01},
    {{-3.37163666937775774e-01, -2.52138530596949795e-01, -2.46310411963512277e-01, -5.42422418400644937e-02,
      2.67546354036343470e-01, -1.12359191313233468e-02, -5.50416436017386462e-02, -2.85989634760784428e-01,
      2.84276261266771879e+00, 2.28640609057066690e+00},
     2.66184683719140058e-01},
    {{-3.23804724610474881e-01, -3.00486639537123124e-01, 5.97989718749250988e-03, -6.04430805086655781e-02,
      4.52291486900478046e-01, -1.28875868013209188e-01, 2.97368471773662213e-01, -4.54258534668076253e-01,
      1.76762766759557954e+00, 2.45978651843712059e+00},
     2.56523531597976584e-01},
    {{-3.24243365381103932e-01, -2.97416126379326851e-01, -4.37756057492964573e-04, -5.31079725716148351e-02,
      4.34420128220554647e-01, -1.20145510920309007e-01, 2.90312460934978034e-01, -4.50465697453917124e-01,
      1.84870917391618450e+00, 2.46748132273880882e+00},
     2.56184414070271038e-01},
};

}  // namespace

extern "C" int mr_predict_speedup(int model, const double* r, double* out)
{
    if (model < 0 || model > 3 || !r || !out) return MR_ERR_INVALID_ARG;
    const RidgeModel& m = kModels[model];
    double v = m.intercept;
    for (int i = 0; i < 10; ++i) v += m.coef[i] * r[i];
    const double s = std::exp(v);
    *out = s;
    if (!std::isfinite(s) || s <= 0.0) return MR_ERR_PREDICT;
    return MR_OK;
}
