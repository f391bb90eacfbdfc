// r2r_pass.cuh -- one axis pass of a 3-D r2r transform over an nx*ny*nz field
// (layout idx = (i*ny + j)*nz + k, the reference's x-slab order, z contiguous).
//
// A CTA owns a tile of W lines: for the z axis W consecutive rows (contiguous), for the
// y and x axes W consecutive k-columns (so every global access is a coalesced run along
// z).  The tile is staged in shared memory as W/2 complex lines, transformed, and written
// back.  The first pass of a 3-D transform reads through a Loader functor (it computes the
// transform input from any number of fields: nonlinearity, spectral update, index-shifted
// gradient spectra, Stokes projection ...); the last pass writes through a Storer functor.
// Passes are in place on the tile, so a 3-D transform needs one scratch field.
#pragma once

#include <type_traits>

#include "fft_tile.cuh"

namespace smadft {

// Element index inside one field: grids are at most 1024 per axis, so every index
// (< 1024^3 = 2^30) fits 32 bits, which keeps the per-element address arithmetic 32-bit.
using idx_t = int;

struct Geom {
    int nx, ny, nz;
    int nyz;         // ny * nz
#ifdef SMADFT_CHECK_BOUNDS
    long long nelem = 0;   // valid element indices [0, nelem) of the pass's fields
    int *chk = nullptr;    // device word set to 1 by the first out-of-range index
#endif
};

// Bounds-check build (-DSMADFT_CHECK_BOUNDS, `make check`): every element index a pass kernel
// hands to its loader or storer is checked against the field size; an index outside it sets
// the context's check word and the access is skipped (loads give zero), so a wrong index
// shows up as a status instead of a memory fault.  In the normal build the check is `true`.
#ifdef SMADFT_CHECK_BOUNDS
__device__ __forceinline__ bool idx_ok(const Geom &g, long long q, int span = 1)
{
    if (q >= 0 && q + span <= g.nelem) return true;
    if (g.chk) atomicCAS(g.chk, 0, 1);
    return false;
}
#else
__device__ __forceinline__ constexpr bool idx_ok(const Geom &, long long, int = 1) { return true; }
#endif

template <typename T>
struct PassArgs {
    Geom g;
    int axis;        // 0 = x, 1 = y, 2 = z
    int kind;        // R2RKind
    int W;           // lines per tile (even)
    int ld;          // shared-memory line stride (complex elements)
    int tiles_b;     // tiles along the second tile coordinate
    LinePlan<T> P;
};

// Element coordinates for tile-local (t = position along the line, w = line in tile).
struct ElemPos {
    long long idx;
    int i, j, k;
    bool valid;
};

template <typename T>
__device__ __forceinline__ ElemPos elem_pos(const PassArgs<T> &a, int t, int w)
{
    ElemPos e;
    const Geom &g = a.g;
    if (a.axis == 2) {
        long long line = (long long)blockIdx.x * a.W + w;    // line = i*ny + j
        e.valid = line < (long long)g.nx * g.ny;
        int i = (int)(line / g.ny);
        int j = (int)(line - (long long)i * g.ny);
        e.i = i; e.j = j; e.k = t;
        e.idx = line * g.nz + t;
    } else {
        const int tb = blockIdx.x % a.tiles_b;
        const int ta = blockIdx.x / a.tiles_b;
        const int k = tb * a.W + w;
        e.valid = k < g.nz;
        e.k = k;
        if (a.axis == 1) {  // lines (i, k), t = j
            e.i = ta; e.j = t;
        } else {            // lines (j, k), t = i
            e.j = ta; e.i = t;
        }
        e.idx = ((long long)e.i * g.ny + e.j) * g.nz + k;
    }
    return e;
}

// V consecutive elements p[idx .. idx+V-1]; for V > 1, idx is a multiple of V and p is
// 16-byte aligned (one 8- or 16-byte access: float2 / float4 / double2).
template <typename T, int V>
__device__ __forceinline__ void vld(const T *__restrict__ p, idx_t idx, T *o)
{
    if constexpr (V == 4 && sizeof(T) == 4) {
        const float4 u = *reinterpret_cast<const float4 *>(p + idx);
        o[0] = u.x; o[1] = u.y; o[2] = u.z; o[3] = u.w;
    } else if constexpr (V == 2 && sizeof(T) == 8) {
        const double2 u = *reinterpret_cast<const double2 *>(p + idx);
        o[0] = u.x; o[1] = u.y;
    } else if constexpr (V == 2 && sizeof(T) == 4) {
        const float2 u = *reinterpret_cast<const float2 *>(p + idx);
        o[0] = u.x; o[1] = u.y;
    } else {
#pragma unroll
        for (int q = 0; q < V; q++) o[q] = p[idx + q];
    }
}

template <typename T, int V>
__device__ __forceinline__ void vst(T *__restrict__ p, idx_t idx, const T *v)
{
    if constexpr (V == 4 && sizeof(T) == 4) {
        *reinterpret_cast<float4 *>(p + idx) = make_float4(v[0], v[1], v[2], v[3]);
    } else if constexpr (V == 2 && sizeof(T) == 8) {
        *reinterpret_cast<double2 *>(p + idx) = make_double2(v[0], v[1]);
    } else if constexpr (V == 2 && sizeof(T) == 4) {
        *reinterpret_cast<float2 *>(p + idx) = make_float2(v[0], v[1]);
    } else {
#pragma unroll
        for (int q = 0; q < V; q++) p[idx + q] = v[q];
    }
}

// V elements of an array of element type S, converted to / from the compute type T (the
// spectral state is FP64 for every compute precision); S == T is vld / vst.
template <typename T, int V, typename S>
__device__ __forceinline__ void vld_as(const S *__restrict__ p, idx_t idx, T *o)
{
    if constexpr (std::is_same<S, T>::value) {
        vld<T, V>(p, idx, o);
    } else {
        S t[V];
        if constexpr (sizeof(S) == 8 && V % 2 == 0) {
#pragma unroll
            for (int h = 0; h < V; h += 2) vld<S, 2>(p, idx + h, t + h);
        } else {
            vld<S, V>(p, idx, t);
        }
#pragma unroll
        for (int q = 0; q < V; q++) o[q] = T(t[q]);
    }
}
template <typename T, int V, typename S>
__device__ __forceinline__ void vst_as(S *__restrict__ p, idx_t idx, const T *v)
{
    if constexpr (std::is_same<S, T>::value) {
        vst<T, V>(p, idx, v);
    } else {
        S t[V];
#pragma unroll
        for (int q = 0; q < V; q++) t[q] = S(v[q]);
        if constexpr (sizeof(S) == 8 && V % 2 == 0) {
#pragma unroll
            for (int h = 0; h < V; h += 2) vst<S, 2>(p, idx + h, t + h);
        } else {
            vst<S, V>(p, idx, t);
        }
    }
}

// Functor interface of the pass kernels.  A loader fills out[0..V-1] with the transform
// input at (i, j, k+u), u < V (memory idx+u, consecutive along z); a storer consumes the
// transform output for the same V elements.  A storer that reads state before writing it
// (the spectral updates) exposes the read as pre() (PRE values per element into buf) and
// the rest as fin(), so kernels can issue the reads of several elements before any write;
// store() = pre() + fin().  The pre() values have the storer's type Pre when it declares
// one (pre_t), else the compute type.  LoadArr / StoreArr move an array of element type S.
template <typename T, typename S = T>
struct LoadArr {
    const S *__restrict__ p;
    template <int V>
    __device__ __forceinline__ void load(idx_t idx, int, int, int, T *out) const { vld_as<T, V, S>(p, idx, out); }
};
template <typename T, typename S = T>
struct StoreArr {
    S *__restrict__ p;
    static constexpr int PRE = 0;
    template <int V>
    __device__ __forceinline__ void pre(idx_t, int, int, int, T *) const {}
    template <int V>
    __device__ __forceinline__ void fin(idx_t idx, int, int, int, const T *v, const T *) const { vst_as<T, V, S>(p, idx, v); }
    template <int V>
    __device__ __forceinline__ void store(idx_t idx, int, int, int, const T *v) const { vst_as<T, V, S>(p, idx, v); }
};

// The same for M equal fields laid out one after another, n elements apart (the pooled
// fields of a batch group): CTA row blockIdx.y works on field blockIdx.y, so one launch with
// gridDim.y = M runs an axis pass over all M fields.
template <typename T, typename S = T>
struct LoadArrM {
    const S *__restrict__ p;
    idx_t n;
    template <int V>
    __device__ __forceinline__ void load(idx_t idx, int, int, int, T *out) const
    {
        vld_as<T, V, S>(p + (size_t)blockIdx.y * n, idx, out);
    }
};
template <typename T, typename S = T>
struct StoreArrM {
    S *__restrict__ p;
    idx_t n;
    static constexpr int PRE = 0;
    template <int V>
    __device__ __forceinline__ void pre(idx_t, int, int, int, T *) const {}
    template <int V>
    __device__ __forceinline__ void fin(idx_t idx, int, int, int, const T *v, const T *) const
    {
        vst_as<T, V, S>(p + (size_t)blockIdx.y * n, idx, v);
    }
    template <int V>
    __device__ __forceinline__ void store(idx_t idx, int, int, int, const T *v) const
    {
        vst_as<T, V, S>(p + (size_t)blockIdx.y * n, idx, v);
    }
};

template <class ST, typename T, class = void>
struct pre_type { using type = T; };
template <class ST, typename T>
struct pre_type<ST, T, std::void_t<typename ST::Pre>> { using type = typename ST::Pre; };
template <class ST, typename T>
using pre_t = typename pre_type<ST, T>::type;

// per-component kinds of the y and z transforms
template <int NC>
struct PlaneKinds {
    int ky[NC], kz[NC];
};

// Loader / storer calls with a component index: multi-component functors (MULTI) take it,
// single ones ignore it.
template <class X, class = void>
struct is_multi : std::false_type {};
template <class X>
struct is_multi<X, std::void_t<decltype(X::MULTI)>> : std::true_type {};

// CTAs per SM a loader's FP32 register-direct pass is sized for: 3 unless the loader says
// otherwise (kMinBlocks; the memory-bound many-field loaders keep more registers at 2)
template <class X, class = void>
struct ld_blocks { static constexpr int value = 3; };
template <class X>
struct ld_blocks<X, std::void_t<decltype(X::kMinBlocks)>> { static constexpr int value = X::kMinBlocks; };

// NC loaders behind one component index (the index is uniform over a CTA)
template <class... L>
struct LoadMulti;
template <class L0>
struct LoadMulti<L0> {
    static constexpr bool MULTI = true;
    static constexpr int kMinBlocks = ld_blocks<L0>::value;
    L0 h;
    template <int V, typename T>
    __device__ __forceinline__ void load(int, idx_t q, int i, int j, int k, T *out) const
    {
        h.template load<V>(q, i, j, k, out);
    }
    // f(loader of component comp): the dispatch happens once, around a whole load loop
    template <class F>
    __device__ __forceinline__ void visit(int, F &&f) const { f(h); }
};
template <class L0, class L1, class... Ls>
struct LoadMulti<L0, L1, Ls...> {
    static constexpr bool MULTI = true;
    static constexpr int kMinBlocks = ld_blocks<L0>::value < ld_blocks<LoadMulti<L1, Ls...>>::value
                                          ? ld_blocks<L0>::value
                                          : ld_blocks<LoadMulti<L1, Ls...>>::value;
    L0 h;
    LoadMulti<L1, Ls...> t;
    template <int V, typename T>
    __device__ __forceinline__ void load(int comp, idx_t q, int i, int j, int k, T *out) const
    {
        if (comp == 0) h.template load<V>(q, i, j, k, out);
        else t.template load<V>(comp - 1, q, i, j, k, out);
    }
    template <class F>
    __device__ __forceinline__ void visit(int comp, F &&f) const
    {
        if (comp == 0) f(h);
        else t.visit(comp - 1, f);
    }
};

// f(ld), or f(loader of component comp) for a multi-component loader
template <class LD, class F>
__device__ __forceinline__ void visit_c(const LD &ld, int comp, F &&f)
{
    if constexpr (is_multi<LD>::value) ld.visit(comp, f);
    else f(ld);
}
template <class L0>
LoadMulti<L0> make_multi(L0 a) { return LoadMulti<L0>{a}; }
template <class L0, class L1, class... Ls>
LoadMulti<L0, L1, Ls...> make_multi(L0 a, L1 b, Ls... r) { return LoadMulti<L0, L1, Ls...>{a, make_multi(b, r...)}; }

// plain stores of component c into field p[c]
template <typename T, int NC>
struct StoreMulti {
    static constexpr bool MULTI = true;
    T *p[NC];
    static constexpr int PRE = 0;
    template <int V>
    __device__ __forceinline__ void pre(int, idx_t, int, int, int, T *) const {}
    template <int V>
    __device__ __forceinline__ void fin(int comp, idx_t idx, int, int, int, const T *v, const T *) const
    {
        vst<T, V>(p[comp], idx, v);
    }
    template <int V>
    __device__ __forceinline__ void store(int comp, idx_t idx, int, int, int, const T *v) const
    {
        vst<T, V>(p[comp], idx, v);
    }
};

// Position along the line of a pass along AXIS, and stores one index up along it: output
// position t goes to t + 1 (`stride` elements further), the last position (t = n - 1) is
// dropped and position 0 is zero-filled.  Spectra of a sine axis stored this way sit at
// their true wavenumber (sine index t is wavenumber t + 1).
template <int AXIS>
__device__ __forceinline__ int line_pos(int i, int j, int k) { return AXIS == 0 ? i : AXIS == 1 ? j : k; }
template <typename T, int V>
__device__ __forceinline__ void vst_up(T *p, idx_t idx, idx_t stride, int t, int n, const T *v)
{
    if (t + 1 < n) vst<T, V>(p, idx + stride, v);
    if (t == 0) {
        T z[V];
#pragma unroll
        for (int u = 0; u < V; u++) z[u] = T(0);
        vst<T, V>(p, idx, z);
    }
}

// StoreMulti whose components in `up` (bit c) store one index up along the pass's line axis
template <typename T, int NC, int AXIS>
struct StoreMultiUp {
    static constexpr bool MULTI = true;
    T *p[NC];
    unsigned up;
    idx_t stride;
    int n;
    static constexpr int PRE = 0;
    template <int V>
    __device__ __forceinline__ void pre(int, idx_t, int, int, int, T *) const {}
    template <int V>
    __device__ __forceinline__ void store(int comp, idx_t idx, int i, int j, int k, const T *v) const
    {
        if (up >> comp & 1u) vst_up<T, V>(p[comp], idx, stride, line_pos<AXIS>(i, j, k), n, v);
        else vst<T, V>(p[comp], idx, v);
    }
    template <int V>
    __device__ __forceinline__ void fin(int comp, idx_t idx, int i, int j, int k, const T *v, const T *) const
    {
        store<V>(comp, idx, i, j, k, v);
    }
};

// one field stored one index up along the pass's line axis (see vst_up)
template <typename T, int AXIS>
struct StoreUp {
    T *p;
    idx_t stride;
    int n;
    static constexpr int PRE = 0;
    template <int V>
    __device__ __forceinline__ void pre(idx_t, int, int, int, T *) const {}
    template <int V>
    __device__ __forceinline__ void store(idx_t idx, int i, int j, int k, const T *v) const
    {
        vst_up<T, V>(p, idx, stride, line_pos<AXIS>(i, j, k), n, v);
    }
    template <int V>
    __device__ __forceinline__ void fin(idx_t idx, int i, int j, int k, const T *v, const T *) const
    {
        store<V>(idx, i, j, k, v);
    }
};

// per-component transform kind of a multi-component pass
template <int NC>
struct KindSet {
    int k[NC];
};

template <int V, class LD, typename T>
__device__ __forceinline__ void load_c(const LD &ld, int comp, idx_t q, int i, int j, int k, T *out)
{
    if constexpr (is_multi<LD>::value) ld.template load<V>(comp, q, i, j, k, out);
    else ld.template load<V>(q, i, j, k, out);
}
template <int V, class ST, typename T>
__device__ __forceinline__ void pre_c(const ST &st, int comp, idx_t q, int i, int j, int k, T *buf)
{
    if constexpr (is_multi<ST>::value) st.template pre<V>(comp, q, i, j, k, buf);
    else st.template pre<V>(q, i, j, k, buf);
}
template <int V, class ST, typename T, typename B>
__device__ __forceinline__ void fin_c(const ST &st, int comp, idx_t q, int i, int j, int k, const T *v,
                                      const B *buf)
{
    if constexpr (is_multi<ST>::value) st.template fin<V>(comp, q, i, j, k, v, buf);
    else st.template fin<V>(q, i, j, k, v, buf);
}
template <int V, class ST, typename T>
__device__ __forceinline__ void store_c(const ST &st, int comp, idx_t q, int i, int j, int k, const T *v)
{
    if constexpr (is_multi<ST>::value) st.template store<V>(comp, q, i, j, k, v);
    else st.template store<V>(q, i, j, k, v);
}


// buffer length for a storer's pre() values of V elements (at least 1)
template <class ST, int V>
constexpr int pre_len() { return ST::PRE * V > 0 ? ST::PRE * V : 1; }

template <typename T, class LD, class ST>
__global__ void __launch_bounds__(256) r2r_pass_kernel(PassArgs<T> a, LD ld, ST st)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<T> *bufA = reinterpret_cast<cpx<T> *>(smem_raw);
    const int n = a.P.n;
    const int W = a.W;
    const int nl = W >> 1;                 // complex lines in the tile
    cpx<T> *bufB = bufA + nl * a.ld;
    T *realA = reinterpret_cast<T *>(bufA);
    const int kind = a.kind;
    const bool fwd = (kind == K_DCT2 || kind == K_DST2);
    const int total = n * W;

    // ---- load: input permutation per kind --------------------------------------------
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
        int t, w;
        if (a.axis == 2) { t = e % n; w = e / n; }
        else { w = e % W; t = e / W; }
        ElemPos p = elem_pos(a, t, w);
        T v = T(0);
        if (p.valid && idx_ok(a.g, p.idx)) ld.template load<1>(p.idx, p.i, p.j, p.k, &v);
        int pos;
        if (kind == K_DCT2) pos = makhoul_pos(t, n);
        else if (kind == K_DST2) { pos = makhoul_pos(t, n); if (t & 1) v = -v; }
        else if (kind == K_DCT3) pos = t;
        else pos = n - 1 - t;
        realA[2 * ((w >> 1) * a.ld + pos) + (w & 1)] = v;
    }
    __syncthreads();

    cpx<T> *res;
    if (fwd) {
        res = fft_lines<T, false>(bufA, bufB, nl, a.ld, a.P);
    } else {
        // DCT-III pre-twiddle: Z_t = V_A[t] + i V_B[t],
        // V[t] = exp(+i pi t/2n) (X_t - i X_{n-t}), X_n = 0
        for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
            const int c = e / n;
            const int t = e - c * n;
            const cpx<T> *L = bufA + c * a.ld;
            cpx<T> xt = L[t];
            cpx<T> xm = (t == 0) ? cpx<T>{T(0), T(0)} : L[n - t];
            bufB[c * a.ld + t] = dct3_pre(xt, xm, a.P.h[t]);
        }
        __syncthreads();
        res = fft_lines<T, true>(bufB, bufA, nl, a.ld, a.P);
    }

    // ---- store: output permutation / post-twiddle per kind --------------------------
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
        int o, w;
        if (a.axis == 2) { o = e % n; w = e / n; }
        else { w = e % W; o = e / W; }
        ElemPos p = elem_pos(a, o, w);
        const cpx<T> *L = res + (w >> 1) * a.ld;
        T v;
        if (fwd) {
            const int k = (kind == K_DCT2) ? o : (n - 1 - o);
            cpx<T> zk = L[k];
            cpx<T> zm = L[k == 0 ? 0 : n - k];
            const cpx<T> o = dct2_post(zk, zm, a.P.h[k]);
            v = (w & 1) ? o.y : o.x;
        } else {
            cpx<T> z = L[makhoul_pos(o, n)];
            v = (w & 1) ? z.y : z.x;
            if (kind == K_DST3 && (o & 1)) v = -v;
        }
        if (p.valid && idx_ok(a.g, p.idx)) st.template store<1>(p.idx, p.i, p.j, p.k, &v);
    }
}

}  // namespace smadft
