// Cross-validation drivers (host interface; see cv.cu).
#pragma once

#include "kernels.cuh"
#include "model.cuh"

namespace fpls {

template <class T>
void cv_regression(int method, const T* predictors, const T* responses,
                   const int* folds, int n, int p, int q, const int* prefixes,
                   int prefix_count, int scaling, int metric,
                   bool store_predictions, double* prediction_output,
                   int* status, double* metrics, double* q2_values,
                   double* rmsd_values, double* observed_r2_values);

template <class T>
void cv_classification(int method, const T* predictors, const int* labels,
                       const int* folds, int n, int p, int classes,
                       const int* prefixes, int prefix_count, int scaling,
                       bool use_lda, bool store_predictions, bool store_scores,
                       int* prediction_output, T* score_output, int* status,
                       double* metrics);

}  // namespace fpls
