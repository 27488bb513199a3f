// Kernel PLS on the device: kernel matrices (linear, RBF, polynomial), their
// double centring, and the predictor preprocessing of the kernel PLS wrapper.
#pragma once

namespace fpls {

// K (n1 x n2) = k(X1[i, :], X2[j, :]) for column-major X1 (n1 x p, ld n1) and
// X2 (n2 x p, ld n2), device memory.  kernel 1: x.y; 2: exp(-gamma |x - y|^2)
// with |x|^2 + |y|^2 - 2 x.y and tiny negative distances (> -1e-10) set to 0;
// 3: (gamma x.y + coef0)^degree.  X1 == X2 (same pointer, n1 == n2) uses the
// symmetric product (upper tiles, mirrored).
void kernel_matrix_device(const double* X1, int n1, const double* X2, int n2, int p, int kernel, double gamma,
                          int degree, double coef0, double* K);

// Kc = ((K - col_means) - row_means) + grand_mean in place for the training
// kernel K (n x n); col_means (n) and the grand mean (one double) on the device.
void center_kernel_train_device(double* K, int n, double* col_means, double* grand_mean);

// Same centring of a test kernel (nt x n) with the training column means and
// grand mean (device) and its own row means.
void center_kernel_test_device(double* Kt, int nt, int n, const double* col_means, const double* grand_mean);

// Predictor preprocessing of the kernel PLS wrapper in place: scaling < 3
// subtracts the column means; scaling 2 divides by the column sd (n - 1), with
// 1 for a zero or non-finite sd.  mX, vX (p) on the device.
void preprocess_kernel_x_device(double* X, int n, int p, int scaling, double* mX, double* vX);

}  // namespace fpls
