#!/bin/bash
# run.sh -- build (if needed) and run one of the four problems on the scout-b200 engine.
# Same flags and meaning as the reference's run.sh (run.sh:19-36, 45-106):
#
#   ./run.sh --problem=mis|coloring|bfs|cc --graph=<graph.egr> --init=<initial_state.txt> \
#            --batch=<batch_folder> [--num-batches=N] [--gpu=ID]
#   ./run.sh --problem=mis|coloring|bfs|cc --sample
#
# --num-batches defaults to the number of *.mtx files in the batch folder; --gpu to 0.
# Environment: NVCC (compiler used by the build), SCOUT_ARCH_FLAG (accepted; the engine is
# written for sm_100a and always built for it), SCOUT_SKIP_COMPACTION=1 (mis: keep the .egr
# untouched), SCOUT_DEVICE_BUDGET_GB (cap on the engine's HBM use).
set -euo pipefail

SCRIPT_DIR="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"

usage() {
    cat >&2 <<EOF
Usage: $0 --problem=mis|coloring|bfs|cc --graph=<graph.egr> --init=<initial_state.txt> --batch=<batch_folder> [--num-batches=N] [--gpu=ID]
       $0 --problem=mis|coloring|bfs|cc --sample

  --problem       mis, coloring, bfs, or cc
  --graph         path to the base graph, as a SCOUT .egr binary CSR file
  --init          path to the initial solution this run seeds from (format depends on --problem)
  --batch         path to a folder of batch files named 1.mtx, 2.mtx, ...
  --num-batches   how many batch files to replay (default: count of *.mtx files in --batch)
  --gpu           CUDA device id to run on (default: 0)
  --sample        use the bundled sample dataset instead of --graph/--init/--batch

Environment overrides:
  NVCC                      nvcc binary used by the build (default: nvcc on PATH)
  SCOUT_ARCH_FLAG           accepted for compatibility; the kernels are written for sm_100a
                            (B200) and always built with -gencode arch=compute_100a,code=sm_100a
  SCOUT_SKIP_COMPACTION=1   mis: skip the end-of-run .egr compaction step
  SCOUT_DEVICE_BUDGET_GB    cap on the HBM the engine may use
EOF
}

PROBLEM=""; GRAPH=""; INIT=""; BATCH=""; NUM_BATCHES=""; GPU="0"; USE_SAMPLE=0
for arg in "$@"; do
    case "$arg" in
        --problem=*)     PROBLEM="${arg#--problem=}" ;;
        --graph=*)       GRAPH="${arg#--graph=}" ;;
        --init=*)        INIT="${arg#--init=}" ;;
        --batch=*)       BATCH="${arg#--batch=}" ;;
        --num-batches=*) NUM_BATCHES="${arg#--num-batches=}" ;;
        --gpu=*)         GPU="${arg#--gpu=}" ;;
        --sample)        USE_SAMPLE=1 ;;
        -h|--help)       usage; exit 0 ;;
        *) echo "ERROR: unrecognized argument: $arg" >&2; usage; exit 1 ;;
    esac
done

case "$PROBLEM" in
    mis)      SAMPLE_INIT="sample_mis.txt" ;;
    coloring) SAMPLE_INIT="sample_colors.txt" ;;
    bfs)      SAMPLE_INIT="sample_bfs.txt" ;;
    cc)       SAMPLE_INIT="sample_components.txt" ;;
    "")       echo "ERROR: --problem=mis|coloring|bfs|cc is required" >&2; usage; exit 1 ;;
    *)        echo "ERROR: --problem must be mis, coloring, bfs, or cc, got '$PROBLEM'" >&2; exit 1 ;;
esac

if [ "$USE_SAMPLE" = "1" ]; then
    SAMPLE="$SCRIPT_DIR/tests/golden/sample"
    GRAPH="${GRAPH:-$SAMPLE/sample.egr}"
    INIT="${INIT:-$SAMPLE/$SAMPLE_INIT}"
    BATCH="${BATCH:-$SAMPLE/batches}"
fi
for v in GRAPH INIT BATCH; do
    if [ -z "${!v}" ]; then
        echo "ERROR: --$(echo $v | tr 'A-Z' 'a-z') is required (or use --sample)" >&2
        usage; exit 1
    fi
done
[ -f "$GRAPH" ] || { echo "ERROR: graph file not found: $GRAPH" >&2; exit 1; }
[ -f "$INIT" ]  || { echo "ERROR: initial-state file not found: $INIT" >&2; exit 1; }
[ -d "$BATCH" ] || { echo "ERROR: batch folder not found: $BATCH" >&2; exit 1; }
if [ -z "$NUM_BATCHES" ]; then
    NUM_BATCHES=$(find "$BATCH" -maxdepth 1 -name '*.mtx' | wc -l | tr -d ' ')
fi

if [ -n "${SCOUT_ARCH_FLAG:-}" ] && [ "$SCOUT_ARCH_FLAG" != "-arch=sm_100a" ]; then
    echo "Note: SCOUT_ARCH_FLAG=$SCOUT_ARCH_FLAG ignored; the engine is built for sm_100a" >&2
fi
BIN="$SCRIPT_DIR/bin/scout_$PROBLEM"
if [ ! -x "$BIN" ]; then
    echo "Building $BIN ..."
    (cd "$SCRIPT_DIR" && python -m scout_b200.build --no-ref)
fi
exec "$BIN" "$GRAPH" "$INIT" "$BATCH" "$NUM_BATCHES" "$GPU"
