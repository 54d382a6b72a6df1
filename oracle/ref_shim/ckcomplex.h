/* Minimal complex type with the members and operators the compiled reference
 * leaves use (.re/.im, +, -, *, *=, +=, -=, conj, getMagSqr).  Test infrastructure only. */
#pragma once
struct complex {
  double re, im;
  complex() : re(0), im(0) {}
  complex(double r, double i = 0.0) : re(r), im(i) {}
  double getMagSqr() const { return re * re + im * im; }
  complex& operator*=(double s) { re *= s; im *= s; return *this; }
  complex& operator+=(const complex& o) { re += o.re; im += o.im; return *this; }
  complex& operator-=(const complex& o) { re -= o.re; im -= o.im; return *this; }
  complex operator*(double s) const { return complex(re * s, im * s); }
  complex operator*(const complex& o) const {
    return complex(re * o.re - im * o.im, re * o.im + im * o.re);
  }
  complex operator+(const complex& o) const { return complex(re + o.re, im + o.im); }
  complex operator-(const complex& o) const { return complex(re - o.re, im - o.im); }
  complex conj() const { return complex(re, -im); }
};
