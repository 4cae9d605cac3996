// pd_bonds.h -- device neighbour search of libpdcuda.
#pragma once
#include <cuda_runtime.h>

namespace pd {

// Bond lists of n points on the device. dX [3n], ddelta [n], dmask [n] (crack set bits, may
// be null). lo / h / nc describe the cell grid. d_off [n+1] is filled; *d_nbr_out receives
// a cudaMalloc'd array of *nb_out neighbour indices (bond lists sorted by ascending j).
// *dup_out = 1 if two points coincide (the reference raises "point duplicate found").
// downed [n] (may be null): points of the caller's partition; a pair of two points outside
// it gets no bond (halo rows keep only their bonds to owned points).
cudaError_t device_find_bonds_grid(long long n, const double* dX, const double* ddelta,
                                   const unsigned short* dmask, const unsigned char* downed,
                                   const double lo[3], double h,
                                   const long long nc[3], long long* d_off, int** d_nbr_out,
                                   long long* nb_out, int* dup_out, cudaStream_t s);

void launch_bond_props(long long n, const double* dX, const unsigned char* dfp, const long long* doff,
                       const int* dnbr, double* dL, unsigned char* dfpb, cudaStream_t s);

}  // namespace pd
