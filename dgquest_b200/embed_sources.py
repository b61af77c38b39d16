"""Build step: embeds tile_program.h and jit_prelude.cuh as C string
literals (jit_sources.inc) for the runtime compiler. NVRTC gets fixed-width
integer typedefs in place of <cstdint>."""
import sys

TYPEDEFS = ("typedef unsigned char uint8_t; typedef signed char int8_t; typedef unsigned short uint16_t; "
            "typedef short int16_t; typedef unsigned int uint32_t; typedef int int32_t; "
            "typedef unsigned long long uint64_t; typedef long long int64_t;")


def literal(name, text):
    text = text.replace("#include <cstdint>", TYPEDEFS)
    assert ")DGQJ\"" not in text
    return f'static const char *{name} = R"DGQJ({text})DGQJ";\n'


def main(tile_h, prelude_h, out):
    with open(out, "w") as f:
        f.write(literal("kTileProgramSource", open(tile_h).read()))
        f.write(literal("kJitPreludeSource", open(prelude_h).read()))


if __name__ == "__main__":
    main(*sys.argv[1:4])
