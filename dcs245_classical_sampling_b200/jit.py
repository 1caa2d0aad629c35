"""Plan-specialised group kernels.

A fused plan with register runs (``fused.build_fused_plan(..., variant=4 or 12)``) fixes, for
every group, the tile shape, the basis, the coset runs, the activity masks and, per run and step,
everything the register-run kernel (``csrc/runs.cuh``) reads from its arguments and dispatches
on at run time.  ``group_source`` writes one CUDA kernel per group with all of that as
constants (device header ``csrc/runs_jit.cuh``): no dispatch in the step loop, compile-time
dead masks and partner signs, immediate shared-memory offsets.  ``JitPlan`` compiles the
kernels with NVRTC for sm_100a through the library (``dcs_jit_compile``), caches the cubin by
source hash, loads it and launches a group exactly as ``dcs_fused_runs`` would.  Groups without
register runs keep the library kernel.
"""
from __future__ import annotations

import ctypes
import hashlib
import os
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

from . import _lib
from .fused import run_dim

HERE = Path(__file__).resolve().parent
HEADER = HERE / "csrc" / "runs_jit.cuh"
CACHE_DIR = HERE / "_jit_cache"
KERNEL_VERSION = 9  # bump when the generated code changes meaning

ONE_VECTOR = (0, 1, 3, 5, 7)


def _u64(x):
    return f"{int(x) & 0xFFFFFFFFFFFFFFFF}ull"


def _beff(kind, ts, R, ptab, touched=False):
    """The step's sign functional on the local bits.  The step's own bits are dropped when every
    representative has them clear (no basis vector touching the role); with touching bases a
    representative may have them set, so they stay."""
    bl = sum(((ptab >> (1 << k)) & 1) << k for k in range(R))
    if touched:
        return bl
    own = 0
    if kind in ONE_VECTOR:
        own = 1 << int(ts["rk1"])
    elif kind == 6:
        own = (1 << int(ts["rk1"])) | (1 << int(ts["rk2"]))
    return bl & ~own


def _deposit_expr(g, var="tile"):
    terms = []
    for r in range(int(g["ncoset_runs"])):
        w = int(g["coset_runs"][r])
        src, dst, ln = w & 255, (w >> 8) & 255, (w >> 16) & 255
        mask = (1 << 64) - 1 if ln >= 64 else (1 << ln) - 1
        terms.append(f"((({var} >> {src}) & {_u64(mask)}) << {dst})")
    return " | ".join(terms) if terms else "0ull"


def _group_runs(fp, gi):
    """[(first step within the group, step count)] of the register runs of group gi."""
    g = fp.groups[gi]
    first, count = int(g["first"]), int(g["count"])
    out, s = [], 0
    while s < count:
        n = int(fp.tile_steps[first + s]["run_len"])
        if n < 1:
            raise ValueError(f"group {gi}: malformed run at step {first + s}")
        out.append((s, n))
        s += n
    return out


def uses_tile_buffer(fp, gi):
    """False when the group's kernel keeps no tile in shared memory (direct I/O, one run)."""
    return not (getattr(fp, "direct_io", True) and len(_group_runs(fp, gi)) == 1
                and _direct_ok(fp, gi))


def _direct_ok(fp, gi):
    """Direct I/O needs one coset-skip mask for the whole group (coset slots keep their activity
    inside a group, so this holds for every plan the planner builds)."""
    g = fp.groups[gi]
    first, count = int(g["first"]), int(g["count"])
    return len({int(fp.tile_steps[first + s]["cskip"]) for s in range(count)}) == 1


def _gaddr_fn(g):
    TD, LOW = int(g["tile_dim"]), int(g["low_bits"])
    lowmask = (1 << LOW) - 1
    basis = [int(g["basis"][i]) for i in range(16)]

    def gaddr(t):
        a = t & lowmask
        for i in range(TD - LOW):
            if (t >> (LOW + i)) & 1:
                a ^= basis[i]
        return a
    return gaddr


def pair_bit(offs, R):
    """The local bit whose basis vector is tile bit 0, if every entry with that bit clear sits at
    an even tile offset: local entries j and j | 2^k are then one aligned 16-byte word (complex64).
    A run basis that touches other roles (variant bit 6) may give some of those entries an odd
    offset; then the run moves single entries."""
    k0 = next((k for k in range(R) if int(offs[1 << k]) == 1), None)
    if k0 is None or any(int(offs[j]) & 1 for j in range(1 << R) if not (j >> k0) & 1):
        return None
    return k0


def prefetch_layout(fp, gi, threads=256, kb=None):
    """Staging of the next tile's first-run entries (``fp.prefetch_kb`` > 0): every thread copies
    the entries its own cosets of the next tile will load, asynchronously, into its own slots of
    a staging buffer while the current tile runs; the first run then reads them from shared
    memory.  Applies to multi-run groups with direct I/O whose first-run entries are live at the
    same local indices in every coset (the address of every free tile coordinate avoids the
    inactive slots).  Returns None, or the layout: KPF staged loop iterations (as many as fit
    in prefetch_kb), the staged units (16-byte pairs (j, j1) or single entries (j, None)), the
    unit size UB, the slot stride NBT (threads of the first run) and the staging bytes."""
    kb = int((getattr(fp, "prefetch_kb", 0) if kb is None else kb) or 0)
    if kb <= 0 or not getattr(fp, "direct_io", True) or not _direct_ok(fp, gi) or not uses_tile_buffer(fp, gi):
        return None
    if getattr(fp, "coset_pairs", False):
        return None
    g = fp.groups[gi]
    if not int(g["variant"]) & 4 or packable(fp, gi):
        return None
    fp64 = bool(getattr(fp, "fp64", False))
    R = run_dim(int(g["variant"]))
    first = int(g["first"])
    TD, LOW = int(g["tile_dim"]), int(g["low_bits"])
    T = 1 << TD
    lognt = threads.bit_length() - 1
    in_mask = int(fp.dsteps[first]["in_mask"])
    in_inact = ~in_mask & 0xFFFFFFFFFFFFFFFF
    gaddr = _gaddr_fn(g)
    s, _ = _group_runs(fp, gi)[0]
    tr = fp.tile_runs[first + s]
    nins = int(tr["nins"])
    ins = [int(x) for x in tr["ins"][:nins]]
    NB = T >> nins
    niter = NB >> lognt if NB > threads else 1
    free = [b for b in range(TD) if b not in ins]
    if any(gaddr(1 << f) & in_inact for f in free):
        return None
    G = [gaddr(int(fp.run_off[first + s][j])) for j in range(1 << R)]
    live = [j for j in range(1 << R) if not G[j] & in_inact]
    if not live:
        return None
    k0 = None if fp64 else pair_bit(fp.run_off[first + s], R)
    pair_in = LOW >= 1 and (in_mask & 1)
    if k0 is not None and pair_in:
        units = [(j, j | (1 << k0)) for j in live if not (j >> k0) & 1]
        UB = 16
    else:
        units = [(j, None) for j in live]
        UB = 16 if fp64 else 8
    NBT = min(NB, threads)
    per_iter = len(units) * UB * NBT
    KPF = min(niter, (kb * 1024) // per_iter)
    if KPF < 1:
        return None
    return {"KPF": KPF, "niter": niter, "units": units, "UB": UB, "NBT": NBT, "NB": NB, "ins": ins,
            "G": G, "stg_bytes": KPF * per_iter}


def _split_bits(TD, LOW):
    nbits = max(1, TD - LOW)
    return nbits, nbits // 2


def group_smem(fp, gi, threads=256, kb=None):
    """Dynamic shared memory of the kernel of group gi: the tile buffer (if the kernel keeps one),
    the table(s) of high tile-coordinate addresses and the staging buffer (prefetch_layout with
    `kb`, default the plan's prefetch_kb)."""
    g = fp.groups[gi]
    TD, LOW = int(g["tile_dim"]), int(g["low_bits"])
    entry = 16 if getattr(fp, "fp64", False) else 8
    tile = entry * (1 << TD) if uses_tile_buffer(fp, gi) else 0
    lay = prefetch_layout(fp, gi, threads, kb)
    if lay is None:
        return tile + 8 * (1 << (TD - LOW))
    nbits, A = _split_bits(TD, LOW)
    hi = 8 * ((1 << A) + (1 << (nbits - A)))
    return tile + ((hi + 15) // 16) * 16 + lay["stg_bytes"]


def _fixmask(fp, first, count):
    """Bit s: step first + s is a fixed kind (its factor is the weight its y selects)."""
    m = 0
    for s in range(count):
        if int(fp.dsteps[first + s]["kind"]) in (4, 5):  # DCS_KIND_FIXED, DCS_KIND_FIXED_SHRINK
            m |= 1 << s
    return m


def group_source(plan, fp, gi, minb=3, threads=256, kb=None, wait_check=False):
    """CUDA source of the kernel of group gi (``dcs_g<gi>``); None if the group has no runs.

    Direct I/O (``fp.direct_io``, the default): the first run of a tile loads its cosets from
    the table into registers and the last run stores them to the table, scaled, with the max;
    shared memory holds the tile only between runs.  The table address of tile entry t is the
    XOR-linear map addr(t) = (t & lowmask) ^ sum of basis vectors of t's high bits, so entry j of
    the coset of t0 sits at base ^ addr(t0) ^ addr(off_j), the last term a constant of the plan.
    Without it, the tile is staged in shared memory on load and store (the library kernel's
    scheme).  With ``fp.coset_pairs`` a thread takes two cosets per loop iteration where it has
    an even number of them.  `threads` per CTA: a power of two from 128 to 1024 (the packed form
    takes 256 only).

    With ``fp.fp64`` the group runs on a complex128 table with FP64 arithmetic (the unit defines
    DCS_JIT_FP64): entries are 16 bytes, so every entry is one 16-byte access and coset pairs
    along tile bit 0 are not merged; such groups need direct I/O."""
    if threads not in (128, 256, 512, 1024):
        raise ValueError(f"threads {threads}")
    lognt = threads.bit_length() - 1
    coset_pairs = bool(getattr(fp, "coset_pairs", False))
    fp64 = bool(getattr(fp, "fp64", False))
    esh = 4 if fp64 else 3  # log2 of the entry size in bytes
    g = fp.groups[gi]
    if not int(g["variant"]) & 4:
        return None
    if packable(fp, gi):
        if threads != 256:
            raise ValueError("the packed group kernels run 256 threads per CTA")
        return _packed_source(fp, gi, minb)
    direct = bool(getattr(fp, "direct_io", True)) and _direct_ok(fp, gi)
    if fp64 and not direct:
        raise ValueError(f"group {gi}: the complex128 group kernels read and write the table directly")
    R = run_dim(int(g["variant"]))
    first, count = int(g["first"]), int(g["count"])
    TD, LOW = int(g["tile_dim"]), int(g["low_bits"])
    T = 1 << TD
    lowmask = (1 << LOW) - 1
    in_mask = int(fp.dsteps[first]["in_mask"])
    out_mask = int(g["out_mask"])
    in_inact = ~in_mask & 0xFFFFFFFFFFFFFFFF
    out_inact = ~out_mask & 0xFFFFFFFFFFFFFFFF
    pair_in = LOW >= 1 and (in_mask & 1)
    pair_out = LOW >= 1 and (out_mask & 1)
    nb = max(1, TD - LOW)
    basis = [int(g["basis"][i]) for i in range(16)]

    def gaddr(t):
        a = t & lowmask
        for i in range(TD - LOW):
            if (t >> (LOW + i)) & 1:
                a ^= basis[i]
        return a

    runs = _group_runs(fp, gi)
    lay = prefetch_layout(fp, gi, threads, kb) if direct else None
    cskip0 = _u64(fp.tile_steps[first]["cskip"])
    ntiles = _u64(1 << int(g["coset_m"]))
    L = []
    L.append(f"__constant__ uint64_t g{gi}_basis[{nb}] = {{{', '.join(_u64(basis[i]) for i in range(nb))}}};")
    L.append(f"__constant__ uint64_t g{gi}_beta[{count}] = "
             f"{{{', '.join(_u64(fp.dsteps[first + s]['beta']) for s in range(count))}}};")
    L.append(f'extern "C" __global__ void __launch_bounds__({threads}, {minb})')
    L.append(f"dcs_g{gi}(cplx_t* __restrict__ E, const jit_param* __restrict__ params, "
             "unsigned long long* __restrict__ maxbits, jit_scale* __restrict__ scale) {")
    L.append(f"    constexpr int TD = {TD}, LOW = {LOW}, T = 1 << TD, COUNT = {count}, FIRST = {first};")
    L.append("    extern __shared__ __align__(16) unsigned char smem[];")
    if lay is not None:
        nbits, A = _split_bits(TD, LOW)
        hbytes = ((8 * ((1 << A) + (1 << (nbits - A))) + 15) // 16) * 16
        stg_off = (16 if fp64 else 8) * T + hbytes
        L.append("    cplx_t* sh = reinterpret_cast<cplx_t*>(smem);")
        L.append("    uint64_t* hA = reinterpret_cast<uint64_t*>(smem + sizeof(cplx_t) * T);")
        L.append(f"    uint64_t* hB = hA + {1 << A};")
        L.append("    uint64_t* hi_tab = nullptr;")
        L.append(f"    const uint32_t stg_s = (uint32_t)__cvta_generic_to_shared(smem + {stg_off});")
        L.append(f"    jit::fill_hi_split<{nbits}, {A}>(g{gi}_basis, hA, hB);")

        def hexpr(t0):
            sh_ = esh + LOW
            return f"(hA[({t0} >> {sh_}) & {(1 << A) - 1}u] ^ hB[{t0} >> {sh_ + A}])"
    else:
        if uses_tile_buffer(fp, gi):
            L.append("    cplx_t* sh = reinterpret_cast<cplx_t*>(smem);")
            L.append("    uint64_t* hi_tab = reinterpret_cast<uint64_t*>(smem + sizeof(cplx_t) * T);")
        else:
            L.append("    uint64_t* hi_tab = reinterpret_cast<uint64_t*>(smem);")

        def hexpr(t0):
            return f"hi_tab[{t0} >> {esh + LOW}]"
    L.append("    __shared__ wts_t fw[COUNT];")
    L.append("    __shared__ int ovy[COUNT];")
    # Direct I/O: the sign bits alternate between two words, so the barrier after a tile's sign
    # bits is the only one between tiles (the next tile's first shared-memory writes come after
    # it, and warp 0 cannot pass it before every warp has read the previous word).
    L.append("    __shared__ uint32_t cs_sh[2];")
    L.append(f"    const real_t sc = jit::prologue<TD, LOW, COUNT, FIRST, {_fixmask(fp, first, count)}u, "
             f"{'false' if lay is not None else 'true'}>(params, g{gi}_basis, maxbits, {gi}, scale, fw, ovy, hi_tab);")
    L.append("    real_t lm = 0;")
    L.append("    uint32_t par = 0;")
    # between tiles, a split barrier (arrive after a tile's last shared-memory reads, wait before
    # the next tile's first shared-memory writes) instead of a barrier at every tile's start
    tilebar = direct and uses_tile_buffer(fp, gi)
    if tilebar:
        L.append("    __shared__ uint64_t tile_bar;")
        # wait_check (tests only): a phase of 64 tiles' arrivals, which a test plan never completes,
        # so every wait gives up
        L.append(f"    if (threadIdx.x == 0) jit::mbar_init(&tile_bar, {threads * (64 if wait_check else 1)}u);")
        L.append("    __syncthreads();")
        L.append("    uint32_t tile_it = 0;")
    if lay is not None:
        # the first run's thread representative, and the copies of a tile's staged entries
        NBT = lay["NBT"]
        lognbt = NBT.bit_length() - 1
        ub_sh = lay["UB"].bit_length() - 1
        nu = len(lay["units"])
        free0 = [b for b in range(TD) if b not in lay["ins"]]
        mhi0 = sum(1 << b for b in free0[lognt:]) << esh
        L.append(f"    const bool pf_thread = (int)threadIdx.x < {lay['NB']};")
        L.append("    uint32_t tp0 = threadIdx.x;")
        for p in lay["ins"]:
            L.append(f"    tp0 = jit::ins0(tp0, {p});")
        L.append(f"    tp0 <<= {esh};")

        def prefetch(tile_expr, ind):
            out = [f"{ind}if (pf_thread) {{",
                   f"{ind}    const uint64_t pt = {tile_expr};",
                   f"{ind}    if (pt < {ntiles}) {{",
                   f"{ind}        const uint64_t pbase = {_deposit_expr(g, 'pt')};",
                   f"{ind}        if (!(pbase & {cskip0})) {{",
                   f"{ind}            uint32_t ptu = 0;",
                   "#pragma unroll"]
            out.append(f"{ind}            for (int pk = 0; pk < {lay['KPF']}; ++pk) {{")
            out.append(f"{ind}                const uint32_t pt0 = tp0 | ptu;")
            out.append(f"{ind}                ptu = ((ptu | ~{mhi0}u) + 1u) & {mhi0}u;")
            out.append(f"{ind}                const uint64_t pa0 = pbase ^ {hexpr('pt0')} ^ (uint64_t)((pt0 >> {esh}) & "
                       f"{lowmask}u);")
            out.append(f"{ind}                const uint32_t pd = stg_s + ((uint32_t)(pk * {nu}) << {lognbt + ub_sh}) + "
                       f"((uint32_t)threadIdx.x << {ub_sh});")
            for u, (j, _) in enumerate(lay["units"]):
                fn = "cp_async16" if lay["UB"] == 16 else "cp_async8"
                out.append(f"{ind}                jit::{fn}(pd + {u << (lognbt + ub_sh)}u, E + (pa0 ^ {_u64(lay['G'][j])}));")
            out.append(f"{ind}            }}")
            out.append(f"{ind}            jit::cp_async_commit();")
            out.append(f"{ind}        }}")
            out.append(f"{ind}    }}")
            out.append(f"{ind}}}")
            return out
        L.extend(prefetch("(uint64_t)blockIdx.x", "    "))
    L.append(f"    for (uint64_t tile = blockIdx.x; tile < {ntiles}; tile += gridDim.x) {{")
    L.append(f"        const uint64_t base = {_deposit_expr(g)};")
    if tilebar or (direct and not uses_tile_buffer(fp, gi)):  # one-run kernels share no buffer
        L.append(f"        const uint32_t csm = jit::warp_sign_bits<COUNT>(g{gi}_beta, base, ovy);")
    elif direct:
        L.append(f"        jit::sign_bits<COUNT>(g{gi}_beta, base, ovy, &cs_sh[par]);")
        L.append("        __syncthreads();")
    else:
        L.append(f"        jit::load_tile<T, LOW, {'true' if pair_in else 'false'}>(E, sh, hi_tab, base, "
                 f"{_u64(in_inact)});")
        L.append(f"        jit::sign_bits<COUNT>(g{gi}_beta, base, ovy, &cs_sh[par]);")
        L.append('        asm volatile("cp.async.wait_all;\\n" ::: "memory");')
        L.append("        __syncthreads();")
    if not (tilebar or (direct and not uses_tile_buffer(fp, gi))):
        L.append("        const uint32_t csm = cs_sh[par];")
    L.append("        unsigned char* shb = smem;")
    if direct:
        L.append(f"        if (!(base & {_u64(fp.tile_steps[first]['cskip'])})) {{")
    for ri, (s, n) in enumerate(runs):
        src_g = direct and ri == 0
        dst_g = direct and ri == len(runs) - 1
        ts0 = fp.tile_steps[first + s]
        tr = fp.tile_runs[first + s]
        if int(tr["count"]) != n or int(tr["r"]) != R:
            raise ValueError(f"group {gi}: malformed run at step {first + s}")
        nins = int(tr["nins"])
        ins = [int(x) for x in tr["ins"][:nins]]
        NB = T >> nins
        niter = NB >> lognt if NB > threads else 1
        free = [b for b in range(TD) if b not in ins]  # thread index bits fill free[:lognt]
        mhi3 = sum(1 << b for b in free[lognt:]) << esh
        free3 = sum(1 << b for b in free) << esh  # bits a representative's byte offset can have

        def sh_off(c, o, free3=free3):
            """Byte offset of a local entry: t0 ^ o, written t0 + o when o has no bit that t0 can
            have (then the offset is an immediate of the shared-memory access)."""
            return f"(t0{c} + {o}u)" if not (o & free3) else f"(t0{c} ^ {o}u)"
        offs = [int(fp.run_off[first + s][j]) << esh for j in range(1 << R)]
        G = [gaddr(int(fp.run_off[first + s][j])) for j in range(1 << R)]
        L.append(f"        // run: steps {first + s}..{first + s + n - 1}, {NB} cosets of {1 << R} entries"
                 f"{', from the table' if src_g else ''}{', to the table' if dst_g else ''}")
        if not direct:
            L.append(f"        if (!(base & {_u64(ts0['cskip'])})) {{")
        L.append(f"            if ((int)threadIdx.x < {NB}) {{")
        L.append("                uint32_t tp = threadIdx.x;")
        for p in ins:
            L.append(f"                tp = jit::ins0(tp, {p});")
        L.append(f"                tp <<= {esh};")
        L.append("                uint32_t tu = 0;")
        if src_g and lay is not None:
            L.append("                jit::cp_async_wait_all();  // this thread's staged entries of this tile")
        # local bit k0 with basis vector e_0: entries j and j | 2^k0 are one aligned 16-byte word
        # (complex64 entries only)
        k0 = None if fp64 else pair_bit(fp.run_off[first + s], R)
        pairs = [(j, j | (1 << k0)) for j in range(1 << R) if not (j >> k0) & 1] if k0 is not None else None
        cos = ["a", "b"] if coset_pairs and niter % 2 == 0 else ["a"]
        L.append("#pragma unroll 1")
        L.append(f"                for (int k = 0; k < {niter // len(cos)}; ++k) {{")
        for c in cos:
            L.append(f"                    const uint32_t t0{c} = tp | tu;")
            L.append(f"                    tu = ((tu | ~{mhi3}u) + 1u) & {mhi3}u;")
            L.append(f"                    cplx_t v{c}[{1 << R}];")
            if src_g or dst_g:
                L.append(f"                    const uint64_t a0{c} = base ^ {hexpr('t0' + c)} ^ "
                         f"(uint64_t)((t0{c} >> {esh}) & {lowmask}u);")
        staged = src_g and lay is not None
        for c in cos:
            if staged:  # entries staged by this thread's copies (iterations < KPF), else from the table
                if lay["KPF"] < niter:
                    L.append(f"                    if (k < {lay['KPF']}) {{")
                L.append(f"                    const unsigned char* sk = smem + ({stg_off}u + ((uint32_t)(k * {nu}) << "
                         f"{lognbt + ub_sh}) + ((uint32_t)threadIdx.x << {ub_sh}));")
                liveset = set()
                for u, (j, j1) in enumerate(lay["units"]):
                    off = u << (lognbt + ub_sh)
                    if j1 is not None:
                        L.append(f"                    {{ const float4 q = *reinterpret_cast<const float4*>(sk + {off}u); "
                                 f"v{c}[{j}] = make_float2(q.x, q.y); v{c}[{j1}] = make_float2(q.z, q.w); }}")
                        liveset |= {j, j1}
                    else:
                        L.append(f"                    v{c}[{j}] = *reinterpret_cast<const cplx_t*>(sk + {off}u);")
                        liveset.add(j)
                for j in range(1 << R):
                    if j not in liveset:
                        L.append(f"                    v{c}[{j}] = jit::f2((real_t)0, (real_t)0);")
                if lay["KPF"] < niter:
                    L.append("                    } else {")
            if src_g:
                if not staged or lay["KPF"] < niter:
                    if pairs and pair_in:
                        for j, j1 in pairs:
                            L.append(f"                    {{ const uint64_t a = a0{c} ^ {_u64(G[j])}; "
                                     f"if (a & {_u64(in_inact)}) {{ v{c}[{j}] = v{c}[{j1}] = make_float2(0.f, 0.f); }} "
                                     f"else {{ const float4 q = __ldcg(reinterpret_cast<const float4*>(E + a)); "
                                     f"v{c}[{j}] = make_float2(q.x, q.y); v{c}[{j1}] = make_float2(q.z, q.w); }} }}")
                    else:
                        for j in range(1 << R):
                            L.append(f"                    {{ const uint64_t a = a0{c} ^ {_u64(G[j])}; "
                                     f"v{c}[{j}] = (a & {_u64(in_inact)}) ? jit::f2((real_t)0, (real_t)0) : "
                                     "__ldcg(E + a); }")
                if staged and lay["KPF"] < niter:
                    L.append("                    }")
            elif pairs:
                for j, j1 in pairs:
                    L.append(f"                    {{ const float4 q = *reinterpret_cast<const float4*>(shb + "
                             f"{sh_off(c, offs[j])}); v{c}[{j}] = make_float2(q.x, q.y); "
                             f"v{c}[{j1}] = make_float2(q.z, q.w); }}")
            else:
                for j, o in enumerate(offs):
                    L.append(f"                    v{c}[{j}] = *reinterpret_cast<const cplx_t*>(shb + {sh_off(c, o)});")
        if tilebar and dst_g:  # this thread's last reads of the buffer in this tile
            L.append(f"                    if (k == {niter // len(cos) - 1}) jit::mbar_arrive(&tile_bar);")
        for i in range(n):
            si = s + i
            st = fp.tile_steps[first + si]
            kind = int(fp.dsteps[first + si]["kind"])
            dead = int(st["rdead"])
            sk, ska = int(st["sK"]) & 1, int(st["sKa"]) & 1
            k1, k2, mix = int(st["rk1"]), int(st["rk2"]), int(st["rmix"])
            # bases touching other roles (variant bit 6): representative and dead-entry masks
            t1, t2, dp = getattr(fp, "step_touch", {}).get(first + si, (0, 0, 0))
            tch1 = f", {t1}, {dp}u" if (t1 or dp) else ""
            tch0 = f", {dp}u" if dp else ""
            tch4 = f", {t1}, {t2}, {dp}u" if (t1 or t2 or dp) else ""
            B = _beff(kind, st, R, fp.step_ptab[first + si], touched=bool(t1 or t2))
            tb3 = (int(st["tbeta"]) << esh) & 0xFFFFFFFF
            for c in cos:
                m0 = f"(((uint32_t)__popc(t0{c} & {tb3}u) ^ (csm >> {si})) & 1u) << 31"
                args = f"(v{c}, fw[{si}], ovy[{si}] >> 1, {m0})"
                if kind in ONE_VECTOR:
                    call = f"jit::body1<{kind}, {R}, {k1}, {B}, {dead}, {sk}, {ska}{tch1}>{args};"
                elif kind in (2, 4):
                    call = f"jit::body0<{kind}, {R}, {B}, {dead}{tch0}>{args};"
                else:
                    call = f"jit::body4<{R}, {k1}, {k2}, {mix}, {B}, {dead}, {sk}, {ska}{tch4}>{args};"
                L.append(f"                    {call}")
        if tilebar and ri == 0:  # the previous tile's last reads of the buffer are done
            L.append("                    if (tile_it && !jit::mbar_wait(&tile_bar, (tile_it - 1u) & 1u)) "
                     "jit::wait_failed(scale, lm);")
        for c in cos:
            if dst_g:
                if pairs and pair_out:
                    for j, j1 in pairs:
                        L.append(f"                    {{ const uint64_t a = a0{c} ^ {_u64(G[j])}; "
                                 f"if (!(a & {_u64(out_inact)})) {{ const float4 q = make_float4(v{c}[{j}].x * sc, "
                                 f"v{c}[{j}].y * sc, v{c}[{j1}].x * sc, v{c}[{j1}].y * sc); "
                                 "lm = fmaxf(lm, fmaxf(q.x * q.x + q.y * q.y, q.z * q.z + q.w * q.w)); "
                                 "*reinterpret_cast<float4*>(E + a) = q; } }")
                else:
                    for j in range(1 << R):
                        L.append(f"                    {{ const uint64_t a = a0{c} ^ {_u64(G[j])}; "
                                 f"if (!(a & {_u64(out_inact)})) {{ const cplx_t q = jit::f2(v{c}[{j}].x * sc, "
                                 f"v{c}[{j}].y * sc); lm = jit::rmax(lm, jit::norm2(q)); E[a] = q; }} }}")
            elif pairs:
                for j, j1 in pairs:
                    L.append(f"                    *reinterpret_cast<float4*>(shb + {sh_off(c, offs[j])}) = "
                             f"make_float4(v{c}[{j}].x, v{c}[{j}].y, v{c}[{j1}].x, v{c}[{j1}].y);")
            else:
                for j, o in enumerate(offs):
                    L.append(f"                    *reinterpret_cast<cplx_t*>(shb + {sh_off(c, o)}) = v{c}[{j}];")
        L.append("                }")
        if tilebar and dst_g:  # threads without a coset in the last run read nothing of it
            L.append("            } else {")
            L.append("                jit::mbar_arrive(&tile_bar);")
        L.append("            }")
        if src_g and lay is not None:  # every staged entry is in registers: stage the next tile
            L.extend(prefetch("tile + gridDim.x", "            "))
        if not direct:
            L.append("        }")
        if not dst_g:
            L.append("        __syncthreads();")
    if direct:
        if lay is not None or tilebar:  # a skipped tile: stage the next one, arrive for this one
            L.append("        } else {")
            if lay is not None:
                L.extend(prefetch("tile + gridDim.x", "            "))
            if tilebar:
                L.append("            jit::mbar_arrive(&tile_bar);")
        L.append("        }")
        L.append("        par ^= 1u;")
        if tilebar:
            L.append("        ++tile_it;")
    else:
        L.append(f"        lm = jit::store_tile<T, LOW, {'true' if pair_out else 'false'}>(E, sh, hi_tab, base, "
                 f"{_u64(out_inact)}, sc, lm);")
        L.append("        __syncthreads();")
    L.append("    }")
    L.append(f"    jit::block_max(lm, maxbits, {gi + 1});")
    L.append("}")
    return "\n".join(L) + "\n"


def packable(fp, gi):
    """Packed form for group gi: the plan asks for it (variant bit 1), direct I/O applies, and no
    run of the group has tile bit 0 in its space or among its coset zero bits."""
    g = fp.groups[gi]
    v = int(g["variant"])
    if getattr(fp, "fp64", False) or v & 80:  # the packed bodies: FP32x2, runs up to dimension 4, no touching bases
        return False
    if not (v & 2 and v & 4) or not getattr(fp, "direct_io", True) or not _direct_ok(fp, gi):
        return False
    R = run_dim(v)
    first = int(g["first"])
    if int(g["tile_dim"]) < 1:
        return False
    for s, _ in _group_runs(fp, gi):
        tr = fp.tile_runs[first + s]
        nins = int(tr["nins"])
        if nins >= int(g["tile_dim"]) or (nins and int(tr["ins"][0]) == 0):
            return False
        if any(int(fp.run_off[first + s][j]) & 1 for j in range(1 << R)):
            return False
    return True


def _packed_source(fp, gi, minb):
    """Packed FP32x2 form of group gi: a thread takes the coset pair (t0, t0 | 1) as the two lanes
    of its float2 values (runs_jit.cuh pbody*).  Between runs the tile sits in shared memory as
    (re_2i, re_2i+1, im_2i, im_2i+1) per entry pair, one 16-byte word per local entry of a pair;
    the first run reads the table and the last one writes it (direct I/O)."""
    g = fp.groups[gi]
    R = run_dim(int(g["variant"]))
    first, count = int(g["first"]), int(g["count"])
    TD, LOW = int(g["tile_dim"]), int(g["low_bits"])
    T = 1 << TD
    lowmask = (1 << LOW) - 1
    in_mask = int(fp.dsteps[first]["in_mask"])
    out_mask = int(g["out_mask"])
    in_inact = ~in_mask & 0xFFFFFFFFFFFFFFFF
    out_inact = ~out_mask & 0xFFFFFFFFFFFFFFFF
    nb = max(1, TD - LOW)
    basis = [int(g["basis"][i]) for i in range(16)]

    def gaddr(t):
        a = t & lowmask
        for i in range(TD - LOW):
            if (t >> (LOW + i)) & 1:
                a ^= basis[i]
        return a

    runs = _group_runs(fp, gi)
    L = []
    L.append(f"__constant__ uint64_t g{gi}_basis[{nb}] = {{{', '.join(_u64(basis[i]) for i in range(nb))}}};")
    L.append(f"__constant__ uint64_t g{gi}_beta[{count}] = "
             f"{{{', '.join(_u64(fp.dsteps[first + s]['beta']) for s in range(count))}}};")
    L.append(f'extern "C" __global__ void __launch_bounds__(256, {minb})')
    L.append(f"dcs_g{gi}(float2* __restrict__ E, const jit_param* __restrict__ params, "
             "unsigned long long* __restrict__ maxbits, jit_scale* __restrict__ scale) {")
    L.append(f"    constexpr int TD = {TD}, LOW = {LOW}, T = 1 << TD, COUNT = {count}, FIRST = {first};")
    L.append("    extern __shared__ __align__(16) unsigned char smem[];")
    if len(runs) > 1:
        L.append("    uint64_t* hi_tab = reinterpret_cast<uint64_t*>(smem + sizeof(float2) * T);")
    else:
        L.append("    uint64_t* hi_tab = reinterpret_cast<uint64_t*>(smem);")
    L.append("    __shared__ float4 fw[COUNT];")
    L.append("    __shared__ int ovy[COUNT];")
    L.append("    __shared__ uint32_t cs_sh[2];")
    L.append(f"    const float sc = jit::prologue<TD, LOW, COUNT, FIRST, {_fixmask(fp, first, count)}u>(params, "
             f"g{gi}_basis, maxbits, {gi}, scale, fw, ovy, hi_tab);")
    L.append("    float lm = 0.f;")
    L.append("    uint32_t par = 0;")
    L.append(f"    for (uint64_t tile = blockIdx.x; tile < {_u64(1 << int(g['coset_m']))}; tile += gridDim.x) {{")
    L.append(f"        const uint64_t base = {_deposit_expr(g)};")
    L.append(f"        jit::sign_bits<COUNT>(g{gi}_beta, base, ovy, &cs_sh[par]);")
    L.append("        __syncthreads();")
    L.append("        const uint32_t csm = cs_sh[par];")
    L.append("        unsigned char* shb = smem;")
    L.append(f"        if (!(base & {_u64(fp.tile_steps[first]['cskip'])})) {{")
    for ri, (s, n) in enumerate(runs):
        src_g = ri == 0
        dst_g = ri == len(runs) - 1
        tr = fp.tile_runs[first + s]
        nins = int(tr["nins"])
        ins = [int(x) for x in tr["ins"][:nins]]
        NB2 = T >> (nins + 1)
        niter = NB2 >> 8 if NB2 > 256 else 1
        mhi = int(tr["mhi"])
        mhi3 = (mhi & (mhi - 1)) << 3  # tile bit 0 is the lane bit
        offs = [int(fp.run_off[first + s][j]) << 3 for j in range(1 << R)]
        G = [gaddr(int(fp.run_off[first + s][j])) for j in range(1 << R)]
        L.append(f"        // run: steps {first + s}..{first + s + n - 1}, {NB2} coset pairs of {1 << R} entries"
                 f"{', from the table' if src_g else ''}{', to the table' if dst_g else ''}")
        L.append(f"            if ((int)threadIdx.x < {NB2}) {{")
        L.append("                uint32_t tp = threadIdx.x << 1;")
        for p in ins:
            L.append(f"                tp = jit::ins0(tp, {p});")
        L.append("                tp <<= 3;")
        L.append("                uint32_t tu = 0;")
        L.append("#pragma unroll 1")
        L.append(f"                for (int k = 0; k < {niter}; ++k) {{")
        L.append("                    const uint32_t t0 = tp | tu;")
        L.append(f"                    tu = ((tu | ~{mhi3}u) + 1u) & {mhi3}u;")
        L.append(f"                    jit::C2 v[{1 << R}];")
        if src_g or dst_g:
            L.append(f"                    const uint64_t a0 = base ^ hi_tab[t0 >> {3 + LOW}] ^ "
                     f"(uint64_t)((t0 >> 3) & {lowmask}u);")
        for j in range(1 << R):
            if src_g:
                if not in_inact & 1:
                    L.append(f"                    {{ const uint64_t a = a0 ^ {_u64(G[j])}; if (a & {_u64(in_inact)}) "
                             f"v[{j}] = jit::C2{{make_float2(0.f, 0.f), make_float2(0.f, 0.f)}}; else {{ "
                             f"const float4 q = __ldcg(reinterpret_cast<const float4*>(E + a)); "
                             f"v[{j}] = jit::C2{{make_float2(q.x, q.z), make_float2(q.y, q.w)}}; }} }}")
                else:
                    L.append(f"                    {{ const uint64_t a = a0 ^ {_u64(G[j])}; const float2 q = "
                             f"(a & {_u64(in_inact)}) ? make_float2(0.f, 0.f) : __ldcg(E + a); "
                             f"v[{j}] = jit::C2{{make_float2(q.x, 0.f), make_float2(q.y, 0.f)}}; }}")
            else:
                L.append(f"                    {{ const float4 q = *reinterpret_cast<const float4*>(shb + (t0 ^ {offs[j]}u)); "
                         f"v[{j}] = jit::C2{{make_float2(q.x, q.y), make_float2(q.z, q.w)}}; }}")
        for i in range(n):
            si = s + i
            st = fp.tile_steps[first + si]
            kind = int(fp.dsteps[first + si]["kind"])
            B = _beff(kind, st, R, fp.step_ptab[first + si])
            dead = int(st["rdead"])
            sk, ska = int(st["sK"]) & 1, int(st["sKa"]) & 1
            k1, k2, mix = int(st["rk1"]), int(st["rk2"]), int(st["rmix"])
            tb = int(st["tbeta"])
            tb0 = tb & 1
            tb3 = (tb << 3) & 0xFFFFFFFF
            m0 = f"(((uint32_t)__popc(t0 & {tb3}u) ^ (csm >> {si})) & 1u) << 31"
            args = f"(v, fw[{si}], ovy[{si}] >> 1, {m0})"
            if kind in ONE_VECTOR:
                call = f"jit::pbody1<{kind}, {R}, {k1}, {B}, {dead}, {sk}, {ska}, {tb0}>{args};"
            elif kind in (2, 4):
                call = f"jit::pbody0<{kind}, {R}, {B}, {dead}, {tb0}>{args};"
            else:
                call = f"jit::pbody4<{R}, {k1}, {k2}, {mix}, {B}, {dead}, {sk}, {ska}, {tb0}>{args};"
            L.append(f"                    {call}")
        for j in range(1 << R):
            if dst_g:
                if not out_inact & 1:
                    L.append(f"                    {{ const uint64_t a = a0 ^ {_u64(G[j])}; if (!(a & {_u64(out_inact)})) {{ "
                             f"const float4 q = make_float4(v[{j}].re.x * sc, v[{j}].im.x * sc, v[{j}].re.y * sc, "
                             f"v[{j}].im.y * sc); lm = fmaxf(lm, fmaxf(q.x * q.x + q.y * q.y, q.z * q.z + q.w * q.w)); "
                             "*reinterpret_cast<float4*>(E + a) = q; } }")
                else:
                    L.append(f"                    {{ const uint64_t a = a0 ^ {_u64(G[j])}; if (!(a & {_u64(out_inact)})) {{ "
                             f"const float2 q = make_float2(v[{j}].re.x * sc, v[{j}].im.x * sc); "
                             "lm = fmaxf(lm, q.x * q.x + q.y * q.y); E[a] = q; } }")
            else:
                L.append(f"                    *reinterpret_cast<float4*>(shb + (t0 ^ {offs[j]}u)) = make_float4("
                         f"v[{j}].re.x, v[{j}].re.y, v[{j}].im.x, v[{j}].im.y);")
        L.append("                }")
        L.append("            }")
        if not dst_g:
            L.append("        __syncthreads();")
    L.append("        }")
    L.append("        par ^= 1u;")
    L.append("    }")
    L.append(f"    jit::block_max(lm, maxbits, {gi + 1});")
    L.append("}")
    return "\n".join(L) + "\n"


def group_config(group_cfg, gi, minb, threads):
    """(CTAs per SM of the registers, staging KiB or None, threads per CTA) of group gi: its
    entry of group_cfg, (minb, staging KiB) or (minb, staging KiB, threads), else the plan's."""
    c = tuple((group_cfg or {}).get(gi, (minb, None)))
    return (c[0], c[1], c[2] if len(c) > 2 else threads)


def plan_sources(plan, fp, minb=3, parts=8, threads=256, group_cfg=None, wait_check=False):
    """Translation units (source strings) holding the group kernels, spread over `parts` units
    so that NVRTC compiles them in parallel; returns [(source, [group indices])].  group_cfg:
    {group: (CTAs per SM of its registers, staging KiB[, threads per CTA])} overriding minb, the
    plan's prefetch_kb and `threads` for that group (a unit holds kernels of one thread count)."""
    groups = [gi for gi in range(len(fp.groups)) if int(fp.groups[gi]["variant"]) & 4]
    cfg = {gi: group_config(group_cfg, gi, minb, threads) for gi in groups}
    bodies = {gi: group_source(plan, fp, gi, cfg[gi][0], cfg[gi][2], cfg[gi][1], wait_check) for gi in groups}
    out = []
    for nt in sorted({c[2] for c in cfg.values()}):
        mine = [gi for gi in groups if cfg[gi][2] == nt]
        # balance by generated size
        units = [([], 0) for _ in range(max(1, min(parts, len(mine))))]
        for gi in sorted(mine, key=lambda q: -len(bodies[q])):
            k = min(range(len(units)), key=lambda u: units[u][1])
            units[k] = (units[k][0] + [gi], units[k][1] + len(bodies[gi]))
        for gis, _ in units:
            if not gis:
                continue
            src = (f"#define DCS_JIT_THREADS {nt}\n" + ("#define DCS_JIT_WAIT_LIMIT 4096\n" if wait_check else "") +
                   ("#define DCS_JIT_FP64 1\n" if getattr(fp, "fp64", False) else "") +
                   '#include "runs_jit.cuh"\n\n' + "\n".join(bodies[gi] for gi in sorted(gis)))
            out.append((src, sorted(gis)))
    return out


def compile_source(lib, source, name="dcs_plan.cu"):
    """Cubin of one translation unit (NVRTC, sm_100a), cached on disk by source hash."""
    header = HEADER.read_text()
    key = hashlib.sha256(f"{KERNEL_VERSION}\0{header}\0{source}".encode()).hexdigest()[:32]
    path = CACHE_DIR / f"{key}.cubin"
    if path.exists():
        return path.read_bytes()
    img = ctypes.c_void_p()
    size = ctypes.c_size_t()
    log = ctypes.create_string_buffer(1 << 16)
    rc = lib.dcs_jit_compile(source.encode(), name.encode(), header.encode(), b"runs_jit.cuh", 1,
                             ctypes.byref(img), ctypes.byref(size), log, len(log))
    if rc != 0:
        raise _lib.DCSError(rc, lib.dcs_last_error().decode() + "\n" + log.value.decode(errors="replace"))
    data = ctypes.string_at(img.value, size.value)
    lib.dcs_jit_free(img)
    try:
        CACHE_DIR.mkdir(exist_ok=True)
        tmp = path.with_suffix(f".{os.getpid()}.tmp")
        tmp.write_bytes(data)
        os.replace(tmp, path)
    except OSError:
        pass
    return data


def compile_plan(plan, fp, lib=None, minb=3, parts=8, threads=256, group_cfg=None, wait_check=False):
    """[(cubin, [group indices])] for a fused plan (NVRTC in parallel threads)."""
    lib = lib or _lib.load()
    units = plan_sources(plan, fp, minb, parts, threads, group_cfg, wait_check)
    with ThreadPoolExecutor(max_workers=len(units) or 1) as ex:
        images = list(ex.map(lambda u: compile_source(lib, u[0], f"dcs_plan_{u[1][0]}.cu"), units))
    return [(img, gis) for img, (_, gis) in zip(images, units)]


class JitPlan:
    """Loaded group kernels of one fused plan (current CUDA device)."""

    def __init__(self, plan, fp, lib=None, minb=None, parts=8, threads=256, group_cfg=None, wait_check=False):
        """minb: CTAs per SM the registers are sized for (default: 2 if the plan's variant has
        bit 0, else 3).  group_cfg: {group: (minb, staging KiB[, threads])} for groups that
        differ.  wait_check (tests only): every wait between tiles gives up after 4096 polls,
        to check that such a wait ends and reports itself."""
        self.lib = lib or _lib.load()
        self.fp = fp
        self.kernels = {}
        self._libs = []
        self._images = []
        if minb is None:
            minb = 2 if len(fp.groups) and int(fp.groups[0]["variant"]) & 1 else 3
        self.minb = int(minb)
        self.threads = int(threads)
        self.group_cfg = {int(g): tuple(int(x) for x in c) for g, c in (group_cfg or {}).items()}
        sms = self.lib.dcs_sm_count()
        if getattr(fp, "fp64", False):
            missing = [gi for gi in range(len(fp.groups)) if not int(fp.groups[gi]["variant"]) & 4]
            if missing:  # the library's fused kernels store complex64 only
                raise ValueError(f"complex128 fused plan: groups {missing} have no register runs")
        for img, gis in compile_plan(plan, fp, self.lib, minb, parts, self.threads, self.group_cfg, wait_check):
            buf = ctypes.create_string_buffer(img, len(img))
            self._images.append(buf)
            handle = ctypes.c_void_p()
            _lib.check(self.lib.dcs_jit_load(ctypes.cast(buf, ctypes.c_void_p), ctypes.byref(handle)))
            self._libs.append(handle)
            for gi in gis:
                g = fp.groups[gi]
                _, kb, nt = group_config(self.group_cfg, gi, self.minb, self.threads)
                smem = group_smem(fp, gi, nt, kb)
                k = ctypes.c_void_p()
                per_sm = ctypes.c_int()
                _lib.check(self.lib.dcs_jit_kernel(handle, f"dcs_g{gi}".encode(), smem, nt, ctypes.byref(k),
                                                   ctypes.byref(per_sm)))
                grid = min(sms * max(1, per_sm.value), 1 << int(g["coset_m"]))
                self.kernels[gi] = (k, grid, smem, nt)

    def launch(self, table, params, g0, ng, maxbits, scale, stream):
        """Groups [g0, g0 + ng) on `stream` (ints: device pointers); library status."""
        for gi in range(g0, g0 + ng):
            kern = self.kernels.get(gi)
            if kern is None:
                rc = self.fp.launch_library(self.lib, table, params, gi, 1, maxbits, scale, stream)
            else:
                k, grid, smem, nt = kern
                rc = self.lib.dcs_jit_launch(k, grid, nt, smem, table, params, maxbits, scale, stream)
            if rc != 0:
                return rc
        return 0

    def close(self):
        for h in self._libs:
            self.lib.dcs_jit_unload(h)
        self._libs = []
        self.kernels = {}
