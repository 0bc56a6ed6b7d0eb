"""Build oracle/_ref/libprrtc_ref.so from the REFERENCE's own device code (test infrastructure).

The reference library cannot be built here as a whole: its handlers need XLA's
FFI headers (jaxlib is absent) and its collision/FK device functions come from
PyRoFFI (absent).  The sampling, tree-balance, nearest-neighbour, extend,
dynamic-domain, waypoint and connect arithmetic of its planner does not depend
on either, so this recipe compiles exactly those source lines, read from the
reference tree where they lie, inside small harness kernels of this repository:

  cuda-rrtc/CUDA/prrtc_planner.cu:46-83     dynamic-domain radius shrink / grow (CAS loops)
  cuda-rrtc/CUDA/prrtc_planner.cu:144-157   halton_next_runtime
  cuda-rrtc/CUDA/prrtc_planner.cu:748-758   per-block prime shuffle
  cuda-rrtc/CUDA/prrtc_planner.cu:784-788   Halton sample
  cuda-rrtc/CUDA/prrtc_planner.cu:792-823   tree-side balance (all four modes)
  cuda-rrtc/CUDA/prrtc_planner.cu:842-862   nearest-neighbour scan + block reduction
  cuda-rrtc/CUDA/prrtc_planner.cu:864-878   extend / dynamic-domain skip
  cuda-rrtc/CUDA/prrtc_planner.cu:899-904   edge waypoint interpolation
  cuda-rrtc/CUDA/prrtc_planner.cu:975-993   connect step count and vector
  cuda-rrtc/CUDA/prrtc_nearest_neighbor.cu:21-77   standalone NN kernel
  cuda-rrtc/CUDA/prrtc_extend.cu:14-73             standalone extend kernel

nvcc compiles them with the reference's flags (-O3, default FMA contraction), so
the harness outputs are the reference's own device results.  Output goes only to
oracle/_ref/ (git-ignored).  Nothing is copied into the repository.

The reference tree is found at --reference, else $PRRTC_REFERENCE_DIR, else
/root/reference.

Usage: python oracle/ref/build_ref.py [--reference DIR]
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT_DIR = HERE.parent / "_ref"
OUT = OUT_DIR / "libprrtc_ref.so"
DEFAULT_REF = Path(os.environ.get("PRRTC_REFERENCE_DIR", "/root/reference"))

# (file, first line, last line, text that must appear on the first line)
FRAGMENTS = {
    "radius": ("cuda-rrtc/CUDA/prrtc_planner.cu", 46, 83, "prrtc_radius_shrink_atomic"),
    "balance": ("cuda-rrtc/CUDA/prrtc_planner.cu", 792, 823, "const int size_a"),
    "halton": ("cuda-rrtc/CUDA/prrtc_planner.cu", 144, 157, "halton_next_runtime"),
    "primes": ("cuda-rrtc/CUDA/prrtc_planner.cu", 748, 758, "int primes[16]"),
    "sample": ("cuda-rrtc/CUDA/prrtc_planner.cu", 784, 788, "for (int d = 0; d < dim; ++d)"),
    "nn": ("cuda-rrtc/CUDA/prrtc_planner.cu", 842, 862, "float local_min_sq = FLT_MAX"),
    "extend": ("cuda-rrtc/CUDA/prrtc_planner.cu", 864, 878, "if (tid == 0)"),
    "waypoint": ("cuda-rrtc/CUDA/prrtc_planner.cu", 899, 904, "const float t_frac"),
    "connect": ("cuda-rrtc/CUDA/prrtc_planner.cu", 975, 993, "if (tid == 0)"),
    "nn_kernel": ("cuda-rrtc/CUDA/prrtc_nearest_neighbor.cu", 21, 77, "__global__ void prrtc_nearest_neighbor_kernel"),
    "extend_kernel": ("cuda-rrtc/CUDA/prrtc_extend.cu", 14, 73, "__global__ void prrtc_extend_kernel"),
}


def fragment(ref: Path, name: str) -> str:
    rel, a, b, marker = FRAGMENTS[name]
    lines = (ref / rel).read_text().splitlines()
    text = lines[a - 1:b]
    if marker not in text[0]:
        raise RuntimeError(f"{rel}:{a} does not start the expected fragment ({marker!r})")
    return f"// ---- {rel}:{a}-{b}\n" + "\n".join(text) + "\n"


HARNESS = r'''
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>
#include "prrtc_helpers.cuh"

@radius@

@halton@

// Dynamic-domain updates: update i is op[i] (0 shrink, 1 grow) on radii[idx[i]];
// one thread per update (contending CAS loops) or, with sequential, one thread
// applying them in order.
__global__ void h_radius(float* radii, const int* idx, const int* op, int n, float dd_alpha, float dd_radius,
                         float dd_min_radius, int sequential) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int k0 = sequential ? 0 : i, k1 = sequential ? n : i + 1;
    if (sequential && i != 0) return;
    for (int k = k0; k < k1 && k < n; ++k) {
        if (op[k] == 0) prrtc_radius_shrink_atomic(radii, idx[k], dd_alpha, dd_radius, dd_min_radius);
        else prrtc_radius_grow_atomic(radii, idx[k], dd_alpha);
    }
}

// Tree-side balance of explorer bid = blockIdx.x of gridDim.x for n cases:
// sizes [n][2], local_iters [n], vamp_in / tree_out / vamp_out [n][gridDim.x].
__global__ void h_balance(int* sizes, const int* local_iters, const int* vamp_in, int n, int balance_mode,
                          float tree_ratio, int* tree_out, int* vamp_out) {
    if (threadIdx.x != 0) return;
    const int bid = blockIdx.x;
    for (int c = 0; c < n; ++c) {
        int* tree_sizes = sizes + 2 * c;
        const int local_iter = local_iters[c];
        int vamp_tree_id = vamp_in[c * gridDim.x + bid];
        int t_tree_id_sh = -1, o_tree_id_sh = -1;
        {
@balance@
        }
        tree_out[c * gridDim.x + bid] = t_tree_id_sh;
        vamp_out[c * gridDim.x + bid] = vamp_tree_id;
        (void)o_tree_id_sh;
    }
}

__global__ void h_samples(int explorer, int n, int dim, const float* min_vals, const float* max_vals, float* out) {
    if (threadIdx.x != 0) return;
    const int bid = explorer;
    int prime_order[16];
    int halton_st[CONFIG_DIM_MAX];
    float sample_sh[CONFIG_DIM_MAX];
    {
@primes@
    }
    for (int d = 0; d < CONFIG_DIM_MAX; ++d) halton_st[d] = 1;
    for (int k = 0; k < n; ++k) {
@sample@
        for (int d = 0; d < dim; ++d) out[k * dim + d] = sample_sh[d];
    }
}

__global__ void h_prime_order(int explorer, int* out) {
    if (threadIdx.x != 0) return;
    const int bid = explorer;
    int prime_order[16];
@primes@
    for (int d = 0; d < 16; ++d) out[d] = prime_order[d];
}

// One explorer step of the planner for one (tree, sample): NN over comp_t
// nodes, extend, and the blockDim.x waypoints of the extend edge.
__global__ void h_step(const float* t_cfgs, int max_nodes, int dim, int comp_t, const float* sample,
                       const float* t_radii, int dynamic_domain, float step_size,
                       float* out_dsq, int* out_idx, int* out_skip, float* out_cand, float* out_interp) {
    __shared__ float sdata[64];
    __shared__ int sindex_sh[64];
    __shared__ float sample_sh[CONFIG_DIM_MAX];
    __shared__ float cfg_candidate_sh[CONFIG_DIM_MAX];
    __shared__ int nearest_idx_sh;
    __shared__ bool should_skip_sh;
    __shared__ int any_collision_sh;
    const int tid = threadIdx.x;
    if (tid < dim) sample_sh[tid] = sample[tid];
    __syncthreads();
@nn@
    if (tid == 0) { out_dsq[0] = sdata[0]; out_idx[0] = sindex_sh[0]; }
@extend@
    __syncthreads();
    if (tid == 0) {
        out_skip[0] = should_skip_sh ? 1 : 0;
        for (int d = 0; d < dim; ++d) out_cand[d] = cfg_candidate_sh[d];
    }
    if (!should_skip_sh) {
@waypoint@
        for (int d = 0; d < dim; ++d) out_interp[tid * dim + d] = interp[d];
    }
    (void)any_collision_sh;
}

// Connect set-up for a candidate and the other tree's nearest node.
__global__ void h_connect(const float* o_cfgs, int max_nodes, int dim, const float* cand, float cdsq, int cidx,
                          float step_size, int* out_n_ext, float* out_vec) {
    __shared__ float sdata[64];
    __shared__ int sindex_sh[64];
    __shared__ float cfg_candidate_sh[CONFIG_DIM_MAX];
    __shared__ float curr_cfg_sh[CONFIG_DIM_MAX];
    __shared__ float vec_sh[CONFIG_DIM_MAX];
    __shared__ int connect_nearest_idx_sh, n_extensions_sh, extension_parent_sh;
    const int tid = threadIdx.x;
    const int new_idx_sh = 0;
    if (tid == 0) {
        sdata[0] = cdsq; sindex_sh[0] = cidx;
        for (int d = 0; d < dim; ++d) cfg_candidate_sh[d] = cand[d];
    }
    __syncthreads();
@connect@
    __syncthreads();
    if (tid == 0) {
        out_n_ext[0] = n_extensions_sh;
        for (int d = 0; d < dim; ++d) out_vec[d] = vec_sh[d];
    }
    (void)extension_parent_sh; (void)connect_nearest_idx_sh; (void)curr_cfg_sh;
}

@nn_kernel@

@extend_kernel@

extern "C" {
int ref_radius(float* radii, const int* idx, const int* op, int n, float alpha, float r0, float rmin, int sequential,
               void* s) {
    if (n <= 0) return 0;
    h_radius<<<sequential ? 1 : (n + 127) / 128, sequential ? 32 : 128, 0, (cudaStream_t)s>>>(
        radii, idx, op, n, alpha, r0, rmin, sequential);
    return (int)cudaGetLastError();
}
int ref_balance(int* sizes, const int* local_iters, const int* vamp_in, int n, int nblocks, int mode, float ratio,
                int* tree_out, int* vamp_out, void* s) {
    if (n <= 0 || nblocks < 1) return -1;
    h_balance<<<nblocks, 32, 0, (cudaStream_t)s>>>(sizes, local_iters, vamp_in, n, mode, ratio, tree_out, vamp_out);
    return (int)cudaGetLastError();
}
int ref_halton_samples(int explorer, int n, int dim, const float* lo, const float* hi, float* out, void* s) {
    h_samples<<<1, 32, 0, (cudaStream_t)s>>>(explorer, n, dim, lo, hi, out);
    return (int)cudaGetLastError();
}
int ref_prime_order(int explorer, int* out, void* s) {
    h_prime_order<<<1, 32, 0, (cudaStream_t)s>>>(explorer, out);
    return (int)cudaGetLastError();
}
int ref_step(const float* t_cfgs, int max_nodes, int dim, int comp_t, const float* sample, const float* t_radii,
             int dynamic_domain, float step_size, int block, float* out_dsq, int* out_idx, int* out_skip,
             float* out_cand, float* out_interp, void* s) {
    if (block < 1 || block > 64) return -1;
    h_step<<<1, block, 0, (cudaStream_t)s>>>(t_cfgs, max_nodes, dim, comp_t, sample, t_radii, dynamic_domain,
                                             step_size, out_dsq, out_idx, out_skip, out_cand, out_interp);
    return (int)cudaGetLastError();
}
int ref_connect(const float* o_cfgs, int max_nodes, int dim, const float* cand, float cdsq, int cidx,
                float step_size, int* out_n_ext, float* out_vec, void* s) {
    h_connect<<<1, 32, 0, (cudaStream_t)s>>>(o_cfgs, max_nodes, dim, cand, cdsq, cidx, step_size, out_n_ext,
                                              out_vec);
    return (int)cudaGetLastError();
}
// launched as the reference handler does: 16 threads per query (prrtc_nearest_neighbor.cu:116-122)
int ref_nn(const float* tree, int dim, int max_nodes, int tree_size, const float* q, int batch, int* idx,
           float* dist, void* s) {
    const int threads = 16;
    prrtc_nearest_neighbor_kernel<<<batch, threads, threads * (sizeof(float) + sizeof(int)), (cudaStream_t)s>>>(
        tree, q, tree_size, dim, max_nodes, idx, dist);
    return (int)cudaGetLastError();
}
int ref_extend(const float* tree, const int* nearest, const float* samples, float step, int dim, int max_nodes,
               int batch, float* out, int* parents, int* valid, void* s) {
    prrtc_extend_kernel<<<batch, 128, 0, (cudaStream_t)s>>>(tree, nearest, samples, step, dim, max_nodes, out,
                                                             parents, valid);
    return (int)cudaGetLastError();
}
}
'''


def build(ref: Path = DEFAULT_REF, quiet: bool = False) -> Path | None:
    if not (ref / "cuda-rrtc" / "CUDA" / "prrtc_planner.cu").exists():
        if not quiet:
            print(f"reference sources not found under {ref}; skipping", file=sys.stderr)
        return None
    src = HARNESS
    for name in FRAGMENTS:
        src = src.replace(f"@{name}@", fragment(ref, name))
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    with tempfile.TemporaryDirectory() as td:
        cu = Path(td) / "ref_harness.cu"
        cu.write_text(src)
        tmp = OUT.with_suffix(".so.tmp")
        cmd = [nvcc, "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "--shared",
               "-Xcompiler", "-fPIC", "-I", str(ref / "cuda-rrtc" / "CUDA"), "-o", str(tmp), str(cu)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"reference harness build failed:\n{r.stdout}\n{r.stderr}")
        tmp.replace(OUT)
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", type=Path, default=DEFAULT_REF)
    a = ap.parse_args()
    print(build(a.reference))
