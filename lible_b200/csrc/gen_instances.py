"""Writes the per-class kernel instantiation files under lible_b200/csrc/gen/.

Each file holds a small group of classes of one kernel kind, so the build runs in parallel;
inst_table.cu maps (bra pair type, ket pair type) to the launch wrappers.  A quartet class is
instantiated with the larger pair type in the bra; the host swaps bra and ket (and transposes the
output) for the other orientation.  For J/K the classes whose other orientation takes the register
path are also instantiated that way round (shape 2, chosen by the launch autotuner).
"""
import os

PAIR_TYPES = [(0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (2, 2), (3, 0), (3, 1), (3, 2), (3, 3), (4, 0), (5, 0)]
FP32_MAX_TYPE = 9  # mixed precision is instantiated for the l <= 3 classes (cc-pVTZ)


def kinds():
    yield "fwd64", "launchFwd<{la},{lb},{lc},{ld},double>", len(PAIR_TYPES)
    yield "fwd32", "launchFwd<{la},{lb},{lc},{ld},float>", FP32_MAX_TYPE + 1
    yield "d1", "launchD1<{la},{lb},{lc},{ld}>", len(PAIR_TYPES)


# classes per generated file: small groups keep every nvcc invocation short, so a rebuild spreads
# over all cores instead of waiting on the files of the largest bra types
GROUP = {"fwd64": 2, "fwd32": 2, "d1": 3}


def main():
    here = os.path.dirname(os.path.abspath(__file__))
    out = os.path.join(here, "gen")
    os.makedirs(out, exist_ok=True)
    written = []
    table = ['// Generated by gen_instances.py: lookup of class kernels.',
             '#include "../eri_launch_fwd.cuh"', '', 'namespace lible_b200', '{']
    for kind, tmpl, ntypes in kinds():
        launcher = "launchD1" if kind == "d1" else "launchFwd"
        T = {"fwd64": ",double", "fwd32": ",float", "d1": ""}[kind]
        classes = [(bt, kt) for bt in range(ntypes) for kt in range(bt + 1)]
        name_of = lambda bt, kt: f"launch_{kind}_{bt:02d}_{kt:02d}"
        for g in range(0, len(classes), GROUP[kind]):
            part = classes[g:g + GROUP[kind]]
            body = ['// Generated by gen_instances.py: class kernels ' +
                    ", ".join("(%d,%d|%d,%d)" % (PAIR_TYPES[bt] + PAIR_TYPES[kt]) for bt, kt in part) + '.',
                    '#include "../%s"' % ("eri_launch_d1.cuh" if kind == "d1" else "eri_launch_fwd.cuh"),
                    '', 'namespace lible_b200', '{']
            for bt, kt in part:
                la, lb = PAIR_TYPES[bt]
                lc, ld = PAIR_TYPES[kt]
                body += [f'    cudaError_t {name_of(bt, kt)}(const QuartetArgs &a, cudaStream_t s, int n)',
                         '    {', f'        return {launcher}<{la},{lb},{lc},{ld}{T}>(a, s, n);', '    }']
                if kind.startswith("fwd"):
                    # shape variant 1, instantiated only where it differs from the default
                    body += [f'    cudaError_t {name_of(bt, kt)}_v1(const QuartetArgs &a, cudaStream_t s, int n)',
                             '    {', f'        if constexpr (hasShapeVariant<{la},{lb},{lc},{ld}{T}>())',
                             f'            return {launcher}<{la},{lb},{lc},{ld}{T},1>(a, s, n);',
                             '        else', '            return cudaErrorNotSupported;', '    }']
                    # shape 2: the class in the other orientation (ket types above bra types)
                    body += [f'    cudaError_t {name_of(bt, kt)}_f(const QuartetArgs &a, cudaStream_t s, int n)',
                             '    {', f'        if constexpr (hasFlippedShape<{la},{lb},{lc},{ld}{T}>())',
                             f'            return {launcher}<{lc},{ld},{la},{lb}{T}>(a, s, n);',
                             '        else', '            return cudaErrorNotSupported;', '    }']
            body += ['}', '']
            name = f"inst_{kind}_{g // GROUP[kind]:03d}.cu"
            path = os.path.join(out, name)
            text = "\n".join(body)
            if not os.path.exists(path) or open(path).read() != text:
                with open(path, "w") as fh:
                    fh.write(text)
            written.append(name)
        table += [f'    cudaError_t {name_of(bt, kt)}(const QuartetArgs &, cudaStream_t, int);' for bt, kt in classes]
        if kind.startswith("fwd"):
            table += [f'    cudaError_t {name_of(bt, kt)}_v1(const QuartetArgs &, cudaStream_t, int);'
                      for bt, kt in classes]
            table += [f'    cudaError_t {name_of(bt, kt)}_f(const QuartetArgs &, cudaStream_t, int);'
                      for bt, kt in classes]
        cls = lambda bt, kt: "%d,%d,%d,%d%s" % (PAIR_TYPES[bt] + PAIR_TYPES[kt] + (T,))
        for bt in range(ntypes):
            table.append(f'    static const LaunchFn k_{kind}_{bt:02d}[{bt + 1}] = {{' +
                         ", ".join(f"&{name_of(bt, kt)}" for kt in range(bt + 1)) + '};')
            if kind.startswith("fwd"):
                table.append(f'    static const LaunchFn k_{kind}v_{bt:02d}[{bt + 1}] = {{' +
                             ", ".join(f"hasShapeVariant<{cls(bt, kt)}>() ? &{name_of(bt, kt)}_v1 : nullptr"
                                       for kt in range(bt + 1)) + '};')
                table.append(f'    static const LaunchFn k_{kind}f_{bt:02d}[{bt + 1}] = {{' +
                             ", ".join(f"hasFlippedShape<{cls(bt, kt)}>() ? &{name_of(bt, kt)}_f : nullptr"
                                       for kt in range(bt + 1)) + '};')
                for v in (0, 1):
                    table.append(f'    static const int u_{kind}_{v}_{bt:02d}[{bt + 1}] = {{' +
                                 ", ".join(f"workUnit<{cls(bt, kt)},{v}>()" for kt in range(bt + 1)) + '};')
                flip = lambda bt, kt: "%d,%d,%d,%d%s" % (PAIR_TYPES[kt] + PAIR_TYPES[bt] + (T,))
                table.append(f'    static const int u_{kind}_2_{bt:02d}[{bt + 1}] = {{' +
                             ", ".join(f"hasFlippedShape<{cls(bt, kt)}>() ? workUnit<{flip(bt, kt)},0>() : 0"
                                       for kt in range(bt + 1)) + '};')
        if kind.startswith("fwd"):
            for v in (0, 1, 2):
                table.append(f'    static const int *const u_{kind}_{v}[{ntypes}] = {{' +
                             ", ".join(f"u_{kind}_{v}_{bt:02d}" for bt in range(ntypes)) + '};')
            table.append(f'    static const LaunchFn *const k_{kind}v[{ntypes}] = {{' +
                         ", ".join(f"k_{kind}v_{bt:02d}" for bt in range(ntypes)) + '};')
            table.append(f'    static const LaunchFn *const k_{kind}f[{ntypes}] = {{' +
                         ", ".join(f"k_{kind}f_{bt:02d}" for bt in range(ntypes)) + '};')
        table.append(f'    static const LaunchFn *const k_{kind}[{ntypes}] = {{' +
                     ", ".join(f"k_{kind}_{bt:02d}" for bt in range(ntypes)) + '};')
    for kind, _, ntypes in kinds():
        fn = {"fwd64": "lookupFwd64", "fwd32": "lookupFwd32", "d1": "lookupD1"}[kind]
        if kind == "d1":
            table += [f'    LaunchFn {fn}(int bt, int kt)', '    {',
                      f'        if (bt < 0 || bt >= {ntypes} || kt < 0 || kt > bt)',
                      '            return nullptr;', f'        return k_{kind}[bt][kt];', '    }']
        else:
            table += [f'    LaunchFn {fn}(int bt, int kt, int shape)', '    {',
                      f'        if (bt < 0 || bt >= {ntypes} || kt < 0 || kt > bt)',
                      '            return nullptr;',
                      f'        return shape == 2 ? k_{kind}f[bt][kt] : shape ? k_{kind}v[bt][kt] : k_{kind}[bt][kt];',
                      '    }']
    table += ['    int unitFwd(int bt, int kt, bool fp32, int shape)', '    {',
              '        if (bt < 0 || kt < 0 || kt > bt || bt >= (fp32 ? %d : %d))' % (FP32_MAX_TYPE + 1, len(PAIR_TYPES)),
              '            return 0;',
              '        if (shape == 2)',
              '            return fp32 ? u_fwd32_2[bt][kt] : u_fwd64_2[bt][kt];',
              '        if (shape)',
              '            return fp32 ? u_fwd32_1[bt][kt] : u_fwd64_1[bt][kt];',
              '        return fp32 ? u_fwd32_0[bt][kt] : u_fwd64_0[bt][kt];', '    }',
              '    bool hasFwdVariant(int bt, int kt, bool fp32, int shape)', '    {',
              '        return (fp32 ? lookupFwd32(bt, kt, shape) : lookupFwd64(bt, kt, shape)) != nullptr;', '    }']
    table += ['}', '']
    path = os.path.join(out, "inst_table.cu")
    text = "\n".join(table)
    if not os.path.exists(path) or open(path).read() != text:
        with open(path, "w") as fh:
            fh.write(text)
    written.append("inst_table.cu")
    # drop files of an earlier grouping
    for f in os.listdir(out):
        if f.endswith(".cu") and f not in written:
            os.remove(os.path.join(out, f))
    return [os.path.join(out, w) for w in written]


if __name__ == "__main__":
    for p in main():
        print(p)
