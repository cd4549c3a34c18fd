"""Test infrastructure (oracle): the reference's own main program with the
SWE_USE_CUDA switch (the additions listed below), for an end-to-end check that
the C host drives libswe_b200.so unchanged otherwise.

    python patch_main.py <reference>/swe_code/main/main.c _ref/main_cuda.c

The output is a build intermediate under oracle/_ref/ (never committed).  It is
the reference's main.c (swe_code/main/main.c) with these additions, each
inserted at an anchor that must occur exactly once:
  * the library header after the reference's own includes (main.c:13);
  * the switch and swe_cuda_init_psmd(LPSMD) once the patch data exists
    (before the timestepping block, main.c:192);
  * swe_cuda_set_state(H) after each attempt resets H (main.c:297);
  * swe_cuda_rk_substep(rk_val) as the time loop's stage (main.c:337);
  * swe_cuda_get_state(H), which synchronises, before the loop timer stops
    (main.c:371), so verify_output checks the device's result;
  * swe_cuda_finalize() before process_profiling_results (main.c:414).
With SWE_USE_CUDA unset or 0 the program is the reference's CPU path.
"""
import sys

ADDITIONS = [
    ("#include <profiling.h>\n",
     "#include <profiling.h>\n"
     "#ifdef USE_CUDA\n#include <swe_b200.h>\n#endif\n"),
    ("    // -------------------------------- Timestepping ----------------------------------------\n",
     "    int use_cuda = getenv(\"SWE_USE_CUDA\") && atoi(getenv(\"SWE_USE_CUDA\")) == 1;\n"
     "    #ifdef USE_CUDA\n"
     "    if (use_cuda && swe_cuda_init_psmd(LPSMD) != SWE_OK) {\n"
     "        printf(\"swe_cuda_init: %s\\n\", swe_cuda_last_error());\n"
     "        exit(1);\n"
     "    }\n"
     "    #else\n"
     "    if (use_cuda) { printf(\"Executable was not built with USE_CUDA.\\n\"); exit(1); }\n"
     "    #endif\n"
     "    // -------------------------------- Timestepping ----------------------------------------\n"),
    ("        copy_fp_arr(H, H_init, LPSMD->patch_size * 4);\n",
     "        copy_fp_arr(H, H_init, LPSMD->patch_size * 4);\n"
     "        #ifdef USE_CUDA\n"
     "        if (use_cuda && swe_cuda_set_state(H) != SWE_OK) {\n"
     "            printf(\"swe_cuda_set_state: %s\\n\", swe_cuda_last_error());\n"
     "            exit(1);\n"
     "        }\n"
     "        #endif\n"),
    ("            for (int rk_val = 0; rk_val < 4; rk_val++) {\n",
     "            for (int rk_val = 0; rk_val < 4; rk_val++) {\n"
     "                #ifdef USE_CUDA\n"
     "                if (use_cuda) { swe_cuda_rk_substep(rk_val); continue; }\n"
     "                #endif\n"),
    ("        local_timer.t_main[local_timer.attempt] = getTime() - t_start;\n",
     "        #ifdef USE_CUDA\n"
     "        if (use_cuda && swe_cuda_get_state(H) != SWE_OK) {\n"
     "            printf(\"swe_cuda_get_state: %s\\n\", swe_cuda_last_error());\n"
     "            exit(1);\n"
     "        }\n"
     "        #endif\n"
     "        local_timer.t_main[local_timer.attempt] = getTime() - t_start;\n"),
    ("    process_profiling_results();\n",
     "    #ifdef USE_CUDA\n"
     "    if (use_cuda) swe_cuda_finalize();\n"
     "    #endif\n"
     "    process_profiling_results();\n"),
]


def patch(text: str) -> str:
    for anchor, replacement in ADDITIONS:
        n = text.count(anchor)
        if n != 1:
            raise SystemExit(f"anchor found {n} times (expected once): {anchor.strip()!r}")
        text = text.replace(anchor, replacement)
    return text


if __name__ == "__main__":
    src, dst = sys.argv[1], sys.argv[2]
    with open(src) as f:
        out = patch(f.read())
    with open(dst, "w") as f:
        f.write("/* generated by oracle/patch_main.py from the reference's main.c; not a source */\n" + out)
