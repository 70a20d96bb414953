// FP64 mixed-radix FFT for the oracle (test infrastructure only).
//
// The reference transforms with FP64 cuFFT (src/pipeline/fm_demod.cu:359-371,
// src/pipeline/chroma_decode.cu:498-512,603-622,847-850), a closed library.  This
// is an independent FP64 restatement of the discrete Fourier transform with the
// same conventions: forward = sum x[n] e^{-2 pi i kn/N}, inverse unnormalised;
// R2C returns bins 0..N/2; C2R reads bins 0..N/2 as the Hermitian half of a
// spectrum and ignores the imaginary parts of DC and (even N) Nyquist.
// Sizes must be 7-smooth, as every size the reference plans is
// (fm_demod.cu:22-33, chroma_decode.cu:23-34, next_pow2 for the per-line FFT).
#pragma once
#include <cmath>
#include <complex>
#include <cstdlib>
#include <stdexcept>
#include <vector>

namespace oracle {

using cplx = std::complex<double>;

class ComplexFFT {
 public:
  explicit ComplexFFT(int n) : n_(n) {
    if (n < 1) throw std::invalid_argument("fft size");
    int m = n;
    while (m % 4 == 0) { radices_.push_back(4); m /= 4; }
    while (m % 2 == 0) { radices_.push_back(2); m /= 2; }
    for (int p : {3, 5, 7}) while (m % p == 0) { radices_.push_back(p); m /= p; }
    if (m != 1) throw std::invalid_argument("fft size not 7-smooth");
    roots_.resize(n);
    for (int t = 0; t < n; t++) {
      double ang = -2.0 * M_PI * (double)t / (double)n;
      roots_[t] = cplx(std::cos(ang), std::sin(ang));
    }
  }
  int size() const { return n_; }

  // out may alias nothing; work must hold n elements.  inverse = unnormalised +i sign.
  void run(const cplx* in, cplx* out, cplx* work, bool inverse) const {
    const int n = n_;
    // Ping-pong between `out` and `work`; pick the start so the result lands in `out`.
    int stages = (int)radices_.size();
    cplx* bufs[2] = {out, work};
    int cur = (stages % 2 == 0) ? 0 : 1;
    for (int i = 0; i < n; i++) bufs[cur][i] = in[i];
    if (stages == 0) { if (cur != 0) for (int i = 0; i < n; i++) out[i] = work[i]; return; }
    int ns = 1;
    for (int s = 0; s < stages; s++) {
      const int r = radices_[s];
      const cplx* x = bufs[cur];
      cplx* y = bufs[cur ^ 1];
      const int stride = n / r;
      const int tw_step = n / (ns * r);
      for (int j = 0; j < stride; j++) {
        const int k = j % ns;
        cplx v[7];
        for (int q = 0; q < r; q++) v[q] = x[j + q * stride];
        if (k) {
          for (int q = 1; q < r; q++) {
            cplx w = roots_[(size_t)((long long)k * q * tw_step % n)];
            if (inverse) w = std::conj(w);
            v[q] *= w;
          }
        }
        small_dft(v, r, inverse);
        const int base = (j / ns) * ns * r + k;
        for (int q = 0; q < r; q++) y[base + q * ns] = v[q];
      }
      cur ^= 1;
      ns *= r;
    }
  }

 private:
  void small_dft(cplx* v, int r, bool inverse) const {
    if (r == 2) {
      cplx a = v[0], b = v[1];
      v[0] = a + b; v[1] = a - b;
      return;
    }
    if (r == 4) {
      cplx a = v[0], b = v[1], c = v[2], d = v[3];
      cplx s0 = a + c, s1 = a - c, s2 = b + d, s3 = b - d;
      // multiply s3 by -i (forward) or +i (inverse)
      cplx js3 = inverse ? cplx(-s3.imag(), s3.real()) : cplx(s3.imag(), -s3.real());
      v[0] = s0 + s2; v[2] = s0 - s2;
      v[1] = s1 + js3; v[3] = s1 - js3;
      return;
    }
    cplx t[7];
    for (int a = 0; a < r; a++) {
      cplx acc = 0.0;
      for (int b = 0; b < r; b++) {
        int e = (a * b) % r;
        double ang = (inverse ? 2.0 : -2.0) * M_PI * (double)e / (double)r;
        acc += v[b] * cplx(std::cos(ang), std::sin(ang));
      }
      t[a] = acc;
    }
    for (int a = 0; a < r; a++) v[a] = t[a];
  }

  int n_;
  std::vector<int> radices_;
  std::vector<cplx> roots_;
};

// Real transforms of length n on top of ComplexFFT.  Even n uses the
// half-length packing; odd n a full complex transform.
class RealFFT {
 public:
  explicit RealFFT(int n) : n_(n), even_(n % 2 == 0), c_(even_ ? n / 2 : n) {
    if (even_) {
      int h = n / 2;
      tw_.resize(h + 1);
      for (int k = 0; k <= h; k++) {
        double ang = -2.0 * M_PI * (double)k / (double)n;
        tw_[k] = cplx(std::cos(ang), std::sin(ang));
      }
    }
  }
  int size() const { return n_; }
  int bins() const { return n_ / 2 + 1; }
  size_t work_size() const { return (size_t)3 * (even_ ? n_ / 2 + 1 : n_); }

  // x[n] -> X[0..n/2]
  void forward(const double* x, cplx* X, cplx* work) const {
    if (even_) {
      const int h = n_ / 2;
      cplx* z = work;
      cplx* zf = work + h;
      cplx* w2 = work + 2 * h;
      for (int m = 0; m < h; m++) z[m] = cplx(x[2 * m], x[2 * m + 1]);
      c_.run(z, zf, w2, false);
      for (int k = 0; k <= h; k++) {
        cplx a = zf[k % h];
        cplx b = std::conj(zf[(h - k) % h]);
        cplx e = 0.5 * (a + b);
        cplx o = cplx(0.0, -0.5) * (a - b);
        X[k] = e + tw_[k] * o;
      }
    } else {
      cplx* z = work;
      cplx* zf = work + n_;
      cplx* w2 = work + 2 * n_;
      for (int m = 0; m < n_; m++) z[m] = cplx(x[m], 0.0);
      c_.run(z, zf, w2, false);
      for (int k = 0; k < bins(); k++) X[k] = zf[k];
    }
  }

  // X[0..n/2] (Hermitian half) -> x[n], unnormalised.
  void inverse(const cplx* Xin, double* x, cplx* work) const {
    if (even_) {
      const int h = n_ / 2;
      cplx* z = work;
      cplx* zt = work + h;
      cplx* w2 = work + 2 * h;
      // DC and Nyquist are taken as real.
      auto X = [&](int k) -> cplx {
        if (k == 0 || k == h) return cplx(Xin[k].real(), 0.0);
        return Xin[k];
      };
      for (int k = 0; k < h; k++) {
        cplx a = X(k);
        cplx b = std::conj(X(h - k));
        cplx e = a + b;                                   // 2 * E[k]
        cplx o = (a - b) * std::conj(tw_[k]);             // 2 * O[k]
        z[k] = e + cplx(0.0, 1.0) * o;
      }
      c_.run(z, zt, w2, true);
      for (int m = 0; m < h; m++) {
        x[2 * m] = zt[m].real();
        x[2 * m + 1] = zt[m].imag();
      }
    } else {
      cplx* z = work;
      cplx* zt = work + n_;
      cplx* w2 = work + 2 * n_;
      const int nb = bins();
      z[0] = cplx(Xin[0].real(), 0.0);
      for (int k = 1; k < nb; k++) {
        z[k] = Xin[k];
        z[n_ - k] = std::conj(Xin[k]);
      }
      c_.run(z, zt, w2, true);
      for (int m = 0; m < n_; m++) x[m] = zt[m].real();
    }
  }

 private:
  int n_;
  bool even_;
  ComplexFFT c_;
  std::vector<cplx> tw_;
};

}  // namespace oracle
