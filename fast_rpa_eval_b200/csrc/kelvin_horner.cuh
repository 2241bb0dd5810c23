// Generated by gen_kelvin.py: straight-line Horner evaluation of the
// Kelvin-inverted far-field polynomial, degree-graded coefficient packing.
// Do not edit by hand.
#pragma once

namespace frpa {

constexpr int KELVIN_LMAX = 8;
// number of coefficients of degree <= L
__host__ __device__ constexpr int kelvin_count(int L) { return (L + 1) * (L + 2) * (L + 3) / 6; }
// slot of ux^a uy^b uz^c
__host__ __device__ constexpr int kelvin_index(int a, int b, int c) {
  return (a + b + c) * (a + b + c + 1) * (a + b + c + 2) / 6 + a * (a + b + c + 1) - a * (a - 1) / 2 + b;
}

__device__ __forceinline__ void kelvin_horner_0_1(const double *__restrict__ c, const double *ux, const double *uy, const double *uz, double *P) {
  double Q0;
    { const double k = c[0];
      double R0 = k;
      Q0 = R0;
    }
    P[0] = Q0;
}

__device__ __forceinline__ void kelvin_horner_1_1(const double *__restrict__ c, const double *ux, const double *uy, const double *uz, double *P) {
  double Q0;
    { const double k = c[3];
      double R0 = k;
      Q0 = R0;
    }
    P[0] = Q0;
    { const double k = c[2];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[1];
      double R0 = k;
      { const double k2 = c[0];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
}

__device__ __forceinline__ void kelvin_horner_2_1(const double *__restrict__ c, const double *ux, const double *uy, const double *uz, double *P) {
  double Q0;
    { const double k = c[9];
      double R0 = k;
      Q0 = R0;
    }
    P[0] = Q0;
    { const double k = c[8];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[7];
      double R0 = k;
      { const double k2 = c[3];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
    { const double k = c[6];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[5];
      double R0 = k;
      { const double k2 = c[2];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[4];
      double R0 = k;
      { const double k2 = c[1];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[0];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
}

__device__ __forceinline__ void kelvin_horner_3_1(const double *__restrict__ c, const double *ux, const double *uy, const double *uz, double *P) {
  double Q0;
    { const double k = c[19];
      double R0 = k;
      Q0 = R0;
    }
    P[0] = Q0;
    { const double k = c[18];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[17];
      double R0 = k;
      { const double k2 = c[9];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
    { const double k = c[16];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[15];
      double R0 = k;
      { const double k2 = c[8];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[14];
      double R0 = k;
      { const double k2 = c[7];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[3];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
    { const double k = c[13];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[12];
      double R0 = k;
      { const double k2 = c[6];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[11];
      double R0 = k;
      { const double k2 = c[5];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[2];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[10];
      double R0 = k;
      { const double k2 = c[4];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[1];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[0];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
}

__device__ __forceinline__ void kelvin_horner_4_1(const double *__restrict__ c, const double *ux, const double *uy, const double *uz, double *P) {
  double Q0;
    { const double k = c[34];
      double R0 = k;
      Q0 = R0;
    }
    P[0] = Q0;
    { const double k = c[33];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[32];
      double R0 = k;
      { const double k2 = c[19];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
    { const double k = c[31];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[30];
      double R0 = k;
      { const double k2 = c[18];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[29];
      double R0 = k;
      { const double k2 = c[17];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[9];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
    { const double k = c[28];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[27];
      double R0 = k;
      { const double k2 = c[16];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[26];
      double R0 = k;
      { const double k2 = c[15];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[8];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[25];
      double R0 = k;
      { const double k2 = c[14];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[7];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[3];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
    { const double k = c[24];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[23];
      double R0 = k;
      { const double k2 = c[13];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[22];
      double R0 = k;
      { const double k2 = c[12];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[6];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[21];
      double R0 = k;
      { const double k2 = c[11];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[5];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[2];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[20];
      double R0 = k;
      { const double k2 = c[10];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[4];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[1];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[0];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
}

__device__ __forceinline__ void kelvin_horner_5_1(const double *__restrict__ c, const double *ux, const double *uy, const double *uz, double *P) {
  double Q0;
    { const double k = c[55];
      double R0 = k;
      Q0 = R0;
    }
    P[0] = Q0;
    { const double k = c[54];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[53];
      double R0 = k;
      { const double k2 = c[34];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
    { const double k = c[52];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[51];
      double R0 = k;
      { const double k2 = c[33];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[50];
      double R0 = k;
      { const double k2 = c[32];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[19];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
    { const double k = c[49];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[48];
      double R0 = k;
      { const double k2 = c[31];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[47];
      double R0 = k;
      { const double k2 = c[30];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[18];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[46];
      double R0 = k;
      { const double k2 = c[29];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[17];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[9];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
    { const double k = c[45];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[44];
      double R0 = k;
      { const double k2 = c[28];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[43];
      double R0 = k;
      { const double k2 = c[27];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[16];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[42];
      double R0 = k;
      { const double k2 = c[26];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[15];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[8];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[41];
      double R0 = k;
      { const double k2 = c[25];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[14];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[7];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[3];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
    { const double k = c[40];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[39];
      double R0 = k;
      { const double k2 = c[24];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[38];
      double R0 = k;
      { const double k2 = c[23];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[13];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[37];
      double R0 = k;
      { const double k2 = c[22];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[12];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[6];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[36];
      double R0 = k;
      { const double k2 = c[21];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[11];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[5];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[2];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[35];
      double R0 = k;
      { const double k2 = c[20];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[10];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[4];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[1];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[0];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
}

__device__ __forceinline__ void kelvin_horner_6_1(const double *__restrict__ c, const double *ux, const double *uy, const double *uz, double *P) {
  double Q0;
    { const double k = c[83];
      double R0 = k;
      Q0 = R0;
    }
    P[0] = Q0;
    { const double k = c[82];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[81];
      double R0 = k;
      { const double k2 = c[55];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
    { const double k = c[80];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[79];
      double R0 = k;
      { const double k2 = c[54];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[78];
      double R0 = k;
      { const double k2 = c[53];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[34];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
    { const double k = c[77];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[76];
      double R0 = k;
      { const double k2 = c[52];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[75];
      double R0 = k;
      { const double k2 = c[51];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[33];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[74];
      double R0 = k;
      { const double k2 = c[50];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[32];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[19];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
    { const double k = c[73];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[72];
      double R0 = k;
      { const double k2 = c[49];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[71];
      double R0 = k;
      { const double k2 = c[48];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[31];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[70];
      double R0 = k;
      { const double k2 = c[47];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[30];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[18];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[69];
      double R0 = k;
      { const double k2 = c[46];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[29];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[17];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[9];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
    { const double k = c[68];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[67];
      double R0 = k;
      { const double k2 = c[45];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[66];
      double R0 = k;
      { const double k2 = c[44];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[28];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[65];
      double R0 = k;
      { const double k2 = c[43];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[27];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[16];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[64];
      double R0 = k;
      { const double k2 = c[42];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[26];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[15];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[8];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[63];
      double R0 = k;
      { const double k2 = c[41];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[25];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[14];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[7];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[3];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
    { const double k = c[62];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[61];
      double R0 = k;
      { const double k2 = c[40];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[60];
      double R0 = k;
      { const double k2 = c[39];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[24];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[59];
      double R0 = k;
      { const double k2 = c[38];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[23];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[13];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[58];
      double R0 = k;
      { const double k2 = c[37];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[22];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[12];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[6];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[57];
      double R0 = k;
      { const double k2 = c[36];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[21];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[11];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[5];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[2];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[56];
      double R0 = k;
      { const double k2 = c[35];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[20];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[10];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[4];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[1];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[0];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
}

__device__ __forceinline__ void kelvin_horner_7_1(const double *__restrict__ c, const double *ux, const double *uy, const double *uz, double *P) {
  double Q0;
    { const double k = c[119];
      double R0 = k;
      Q0 = R0;
    }
    P[0] = Q0;
    { const double k = c[118];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[117];
      double R0 = k;
      { const double k2 = c[83];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
    { const double k = c[116];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[115];
      double R0 = k;
      { const double k2 = c[82];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[114];
      double R0 = k;
      { const double k2 = c[81];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[55];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
    { const double k = c[113];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[112];
      double R0 = k;
      { const double k2 = c[80];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[111];
      double R0 = k;
      { const double k2 = c[79];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[54];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[110];
      double R0 = k;
      { const double k2 = c[78];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[53];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[34];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
    { const double k = c[109];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[108];
      double R0 = k;
      { const double k2 = c[77];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[107];
      double R0 = k;
      { const double k2 = c[76];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[52];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[106];
      double R0 = k;
      { const double k2 = c[75];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[51];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[33];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[105];
      double R0 = k;
      { const double k2 = c[74];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[50];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[32];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[19];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
    { const double k = c[104];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[103];
      double R0 = k;
      { const double k2 = c[73];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[102];
      double R0 = k;
      { const double k2 = c[72];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[49];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[101];
      double R0 = k;
      { const double k2 = c[71];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[48];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[31];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[100];
      double R0 = k;
      { const double k2 = c[70];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[47];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[30];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[18];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[99];
      double R0 = k;
      { const double k2 = c[69];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[46];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[29];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[17];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[9];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
    { const double k = c[98];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[97];
      double R0 = k;
      { const double k2 = c[68];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[96];
      double R0 = k;
      { const double k2 = c[67];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[45];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[95];
      double R0 = k;
      { const double k2 = c[66];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[44];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[28];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[94];
      double R0 = k;
      { const double k2 = c[65];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[43];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[27];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[16];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[93];
      double R0 = k;
      { const double k2 = c[64];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[42];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[26];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[15];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[8];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[92];
      double R0 = k;
      { const double k2 = c[63];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[41];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[25];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[14];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[7];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[3];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
    { const double k = c[91];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[90];
      double R0 = k;
      { const double k2 = c[62];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[89];
      double R0 = k;
      { const double k2 = c[61];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[40];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[88];
      double R0 = k;
      { const double k2 = c[60];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[39];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[24];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[87];
      double R0 = k;
      { const double k2 = c[59];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[38];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[23];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[13];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[86];
      double R0 = k;
      { const double k2 = c[58];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[37];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[22];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[12];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[6];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[85];
      double R0 = k;
      { const double k2 = c[57];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[36];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[21];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[11];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[5];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[2];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[84];
      double R0 = k;
      { const double k2 = c[56];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[35];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[20];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[10];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[4];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[1];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[0];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
}

__device__ __forceinline__ void kelvin_horner_8_1(const double *__restrict__ c, const double *ux, const double *uy, const double *uz, double *P) {
  double Q0;
    { const double k = c[164];
      double R0 = k;
      Q0 = R0;
    }
    P[0] = Q0;
    { const double k = c[163];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[162];
      double R0 = k;
      { const double k2 = c[119];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
    { const double k = c[161];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[160];
      double R0 = k;
      { const double k2 = c[118];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[159];
      double R0 = k;
      { const double k2 = c[117];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[83];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
    { const double k = c[158];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[157];
      double R0 = k;
      { const double k2 = c[116];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[156];
      double R0 = k;
      { const double k2 = c[115];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[82];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[155];
      double R0 = k;
      { const double k2 = c[114];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[81];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[55];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
    { const double k = c[154];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[153];
      double R0 = k;
      { const double k2 = c[113];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[152];
      double R0 = k;
      { const double k2 = c[112];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[80];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[151];
      double R0 = k;
      { const double k2 = c[111];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[79];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[54];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[150];
      double R0 = k;
      { const double k2 = c[110];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[78];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[53];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[34];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
    { const double k = c[149];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[148];
      double R0 = k;
      { const double k2 = c[109];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[147];
      double R0 = k;
      { const double k2 = c[108];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[77];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[146];
      double R0 = k;
      { const double k2 = c[107];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[76];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[52];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[145];
      double R0 = k;
      { const double k2 = c[106];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[75];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[51];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[33];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[144];
      double R0 = k;
      { const double k2 = c[105];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[74];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[50];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[32];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[19];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
    { const double k = c[143];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[142];
      double R0 = k;
      { const double k2 = c[104];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[141];
      double R0 = k;
      { const double k2 = c[103];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[73];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[140];
      double R0 = k;
      { const double k2 = c[102];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[72];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[49];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[139];
      double R0 = k;
      { const double k2 = c[101];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[71];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[48];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[31];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[138];
      double R0 = k;
      { const double k2 = c[100];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[70];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[47];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[30];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[18];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[137];
      double R0 = k;
      { const double k2 = c[99];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[69];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[46];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[29];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[17];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[9];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
    { const double k = c[136];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[135];
      double R0 = k;
      { const double k2 = c[98];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[134];
      double R0 = k;
      { const double k2 = c[97];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[68];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[133];
      double R0 = k;
      { const double k2 = c[96];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[67];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[45];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[132];
      double R0 = k;
      { const double k2 = c[95];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[66];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[44];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[28];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[131];
      double R0 = k;
      { const double k2 = c[94];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[65];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[43];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[27];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[16];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[130];
      double R0 = k;
      { const double k2 = c[93];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[64];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[42];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[26];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[15];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[8];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[129];
      double R0 = k;
      { const double k2 = c[92];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[63];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[41];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[25];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[14];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[7];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[3];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
    { const double k = c[128];
      double R0 = k;
      Q0 = R0;
    }
    { const double k = c[127];
      double R0 = k;
      { const double k2 = c[91];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[126];
      double R0 = k;
      { const double k2 = c[90];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[62];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[125];
      double R0 = k;
      { const double k2 = c[89];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[61];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[40];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[124];
      double R0 = k;
      { const double k2 = c[88];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[60];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[39];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[24];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[123];
      double R0 = k;
      { const double k2 = c[87];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[59];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[38];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[23];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[13];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[122];
      double R0 = k;
      { const double k2 = c[86];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[58];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[37];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[22];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[12];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[6];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[121];
      double R0 = k;
      { const double k2 = c[85];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[57];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[36];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[21];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[11];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[5];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[2];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    { const double k = c[120];
      double R0 = k;
      { const double k2 = c[84];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[56];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[35];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[20];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[10];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[4];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[1];
        R0 = fma(R0, uz[0], k2);
      }
      { const double k2 = c[0];
        R0 = fma(R0, uz[0], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
    }
    P[0] = fma(P[0], ux[0], Q0);
}

__device__ __forceinline__ void kelvin_eval_1(int lam, const double *__restrict__ c, const double *ux, const double *uy, const double *uz, double *P) {
  switch (lam) {
    case 0: kelvin_horner_0_1(c, ux, uy, uz, P); break;
    case 1: kelvin_horner_1_1(c, ux, uy, uz, P); break;
    case 2: kelvin_horner_2_1(c, ux, uy, uz, P); break;
    case 3: kelvin_horner_3_1(c, ux, uy, uz, P); break;
    case 4: kelvin_horner_4_1(c, ux, uy, uz, P); break;
    case 5: kelvin_horner_5_1(c, ux, uy, uz, P); break;
    case 6: kelvin_horner_6_1(c, ux, uy, uz, P); break;
    case 7: kelvin_horner_7_1(c, ux, uy, uz, P); break;
    case 8: kelvin_horner_8_1(c, ux, uy, uz, P); break;
    default: break;
  }
}

__device__ __forceinline__ void kelvin_horner_0_2(const double *__restrict__ c, const double *ux, const double *uy, const double *uz, double *P) {
  double Q0; double Q1;
    { const double k = c[0];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    P[0] = Q0;
    P[1] = Q1;
}

__device__ __forceinline__ void kelvin_horner_1_2(const double *__restrict__ c, const double *ux, const double *uy, const double *uz, double *P) {
  double Q0; double Q1;
    { const double k = c[3];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    P[0] = Q0;
    P[1] = Q1;
    { const double k = c[2];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[1];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[0];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
}

__device__ __forceinline__ void kelvin_horner_2_2(const double *__restrict__ c, const double *ux, const double *uy, const double *uz, double *P) {
  double Q0; double Q1;
    { const double k = c[9];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    P[0] = Q0;
    P[1] = Q1;
    { const double k = c[8];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[7];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[3];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
    { const double k = c[6];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[5];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[2];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[4];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[1];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[0];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
}

__device__ __forceinline__ void kelvin_horner_3_2(const double *__restrict__ c, const double *ux, const double *uy, const double *uz, double *P) {
  double Q0; double Q1;
    { const double k = c[19];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    P[0] = Q0;
    P[1] = Q1;
    { const double k = c[18];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[17];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[9];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
    { const double k = c[16];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[15];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[8];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[14];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[7];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[3];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
    { const double k = c[13];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[12];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[6];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[11];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[5];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[2];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[10];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[4];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[1];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[0];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
}

__device__ __forceinline__ void kelvin_horner_4_2(const double *__restrict__ c, const double *ux, const double *uy, const double *uz, double *P) {
  double Q0; double Q1;
    { const double k = c[34];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    P[0] = Q0;
    P[1] = Q1;
    { const double k = c[33];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[32];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[19];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
    { const double k = c[31];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[30];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[18];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[29];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[17];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[9];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
    { const double k = c[28];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[27];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[16];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[26];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[15];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[8];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[25];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[14];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[7];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[3];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
    { const double k = c[24];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[23];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[13];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[22];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[12];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[6];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[21];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[11];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[5];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[2];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[20];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[10];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[4];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[1];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[0];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
}

__device__ __forceinline__ void kelvin_horner_5_2(const double *__restrict__ c, const double *ux, const double *uy, const double *uz, double *P) {
  double Q0; double Q1;
    { const double k = c[55];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    P[0] = Q0;
    P[1] = Q1;
    { const double k = c[54];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[53];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[34];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
    { const double k = c[52];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[51];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[33];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[50];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[32];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[19];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
    { const double k = c[49];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[48];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[31];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[47];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[30];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[18];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[46];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[29];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[17];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[9];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
    { const double k = c[45];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[44];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[28];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[43];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[27];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[16];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[42];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[26];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[15];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[8];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[41];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[25];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[14];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[7];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[3];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
    { const double k = c[40];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[39];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[24];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[38];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[23];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[13];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[37];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[22];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[12];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[6];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[36];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[21];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[11];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[5];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[2];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[35];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[20];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[10];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[4];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[1];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[0];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
}

__device__ __forceinline__ void kelvin_horner_6_2(const double *__restrict__ c, const double *ux, const double *uy, const double *uz, double *P) {
  double Q0; double Q1;
    { const double k = c[83];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    P[0] = Q0;
    P[1] = Q1;
    { const double k = c[82];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[81];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[55];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
    { const double k = c[80];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[79];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[54];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[78];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[53];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[34];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
    { const double k = c[77];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[76];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[52];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[75];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[51];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[33];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[74];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[50];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[32];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[19];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
    { const double k = c[73];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[72];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[49];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[71];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[48];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[31];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[70];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[47];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[30];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[18];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[69];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[46];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[29];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[17];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[9];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
    { const double k = c[68];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[67];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[45];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[66];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[44];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[28];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[65];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[43];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[27];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[16];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[64];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[42];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[26];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[15];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[8];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[63];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[41];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[25];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[14];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[7];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[3];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
    { const double k = c[62];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[61];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[40];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[60];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[39];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[24];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[59];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[38];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[23];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[13];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[58];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[37];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[22];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[12];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[6];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[57];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[36];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[21];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[11];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[5];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[2];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[56];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[35];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[20];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[10];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[4];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[1];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[0];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
}

__device__ __forceinline__ void kelvin_horner_7_2(const double *__restrict__ c, const double *ux, const double *uy, const double *uz, double *P) {
  double Q0; double Q1;
    { const double k = c[119];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    P[0] = Q0;
    P[1] = Q1;
    { const double k = c[118];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[117];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[83];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
    { const double k = c[116];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[115];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[82];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[114];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[81];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[55];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
    { const double k = c[113];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[112];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[80];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[111];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[79];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[54];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[110];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[78];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[53];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[34];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
    { const double k = c[109];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[108];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[77];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[107];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[76];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[52];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[106];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[75];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[51];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[33];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[105];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[74];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[50];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[32];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[19];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
    { const double k = c[104];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[103];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[73];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[102];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[72];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[49];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[101];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[71];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[48];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[31];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[100];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[70];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[47];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[30];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[18];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[99];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[69];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[46];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[29];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[17];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[9];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
    { const double k = c[98];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[97];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[68];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[96];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[67];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[45];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[95];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[66];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[44];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[28];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[94];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[65];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[43];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[27];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[16];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[93];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[64];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[42];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[26];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[15];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[8];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[92];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[63];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[41];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[25];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[14];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[7];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[3];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
    { const double k = c[91];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[90];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[62];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[89];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[61];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[40];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[88];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[60];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[39];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[24];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[87];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[59];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[38];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[23];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[13];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[86];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[58];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[37];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[22];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[12];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[6];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[85];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[57];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[36];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[21];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[11];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[5];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[2];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[84];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[56];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[35];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[20];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[10];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[4];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[1];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[0];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
}

__device__ __forceinline__ void kelvin_horner_8_2(const double *__restrict__ c, const double *ux, const double *uy, const double *uz, double *P) {
  double Q0; double Q1;
    { const double k = c[164];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    P[0] = Q0;
    P[1] = Q1;
    { const double k = c[163];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[162];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[119];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
    { const double k = c[161];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[160];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[118];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[159];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[117];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[83];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
    { const double k = c[158];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[157];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[116];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[156];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[115];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[82];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[155];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[114];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[81];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[55];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
    { const double k = c[154];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[153];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[113];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[152];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[112];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[80];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[151];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[111];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[79];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[54];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[150];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[110];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[78];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[53];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[34];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
    { const double k = c[149];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[148];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[109];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[147];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[108];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[77];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[146];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[107];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[76];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[52];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[145];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[106];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[75];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[51];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[33];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[144];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[105];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[74];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[50];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[32];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[19];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
    { const double k = c[143];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[142];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[104];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[141];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[103];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[73];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[140];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[102];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[72];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[49];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[139];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[101];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[71];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[48];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[31];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[138];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[100];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[70];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[47];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[30];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[18];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[137];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[99];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[69];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[46];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[29];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[17];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[9];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
    { const double k = c[136];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[135];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[98];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[134];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[97];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[68];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[133];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[96];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[67];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[45];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[132];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[95];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[66];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[44];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[28];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[131];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[94];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[65];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[43];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[27];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[16];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[130];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[93];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[64];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[42];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[26];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[15];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[8];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[129];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[92];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[63];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[41];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[25];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[14];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[7];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[3];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
    { const double k = c[128];
      double R0 = k;
      double R1 = k;
      Q0 = R0;
      Q1 = R1;
    }
    { const double k = c[127];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[91];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[126];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[90];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[62];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[125];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[89];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[61];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[40];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[124];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[88];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[60];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[39];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[24];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[123];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[87];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[59];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[38];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[23];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[13];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[122];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[86];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[58];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[37];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[22];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[12];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[6];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[121];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[85];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[57];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[36];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[21];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[11];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[5];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[2];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    { const double k = c[120];
      double R0 = k;
      double R1 = k;
      { const double k2 = c[84];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[56];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[35];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[20];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[10];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[4];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[1];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      { const double k2 = c[0];
        R0 = fma(R0, uz[0], k2);
        R1 = fma(R1, uz[1], k2);
      }
      Q0 = fma(Q0, uy[0], R0);
      Q1 = fma(Q1, uy[1], R1);
    }
    P[0] = fma(P[0], ux[0], Q0);
    P[1] = fma(P[1], ux[1], Q1);
}

__device__ __forceinline__ void kelvin_eval_2(int lam, const double *__restrict__ c, const double *ux, const double *uy, const double *uz, double *P) {
  switch (lam) {
    case 0: kelvin_horner_0_2(c, ux, uy, uz, P); break;
    case 1: kelvin_horner_1_2(c, ux, uy, uz, P); break;
    case 2: kelvin_horner_2_2(c, ux, uy, uz, P); break;
    case 3: kelvin_horner_3_2(c, ux, uy, uz, P); break;
    case 4: kelvin_horner_4_2(c, ux, uy, uz, P); break;
    case 5: kelvin_horner_5_2(c, ux, uy, uz, P); break;
    case 6: kelvin_horner_6_2(c, ux, uy, uz, P); break;
    case 7: kelvin_horner_7_2(c, ux, uy, uz, P); break;
    case 8: kelvin_horner_8_2(c, ux, uy, uz, P); break;
    default: break;
  }
}

// kelvin_eval<N>: N points at a time
template <int N>
__device__ __forceinline__ void kelvin_eval(int lam, const double *__restrict__ c, const double *ux, const double *uy, const double *uz, double *P);
template <>
__device__ __forceinline__ void kelvin_eval<1>(int lam, const double *__restrict__ c, const double *ux, const double *uy, const double *uz, double *P) {
  kelvin_eval_1(lam, c, ux, uy, uz, P);
}
template <>
__device__ __forceinline__ void kelvin_eval<2>(int lam, const double *__restrict__ c, const double *ux, const double *uy, const double *uz, double *P) {
  kelvin_eval_2(lam, c, ux, uy, uz, P);
}

}  // namespace frpa
