#!/usr/bin/env bash
# Regenerates tests/golden/reference_bifurcation/ with the REFERENCE's own
# preprocessing chain (mesher -> spline extractor -> packer), built from the
# reference sources, on a Y-shaped skeleton: the spline extraction at the
# bifurcation has extraordinary vertices, whose elements carry 80 basis
# functions (the most the reference's CUDA path accepts).  Run here (where the
# reference is mounted), never on the GPU box; the committed .xz fixtures are
# what the tests read.
#
#   tubular_mesh pipeline CASE TEMPLATES   preprocessing/mesh/src/main.cpp:152-207
#   spline CASE/ --no-legacy-text          preprocessing/spline/main.cpp
#   iga_pack CASE 1 OUT.ntiga              solvers/cpu/src/iga_pack.cpp:278-417
set -euo pipefail
REF=${REF:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
STUB=$(cd "$HERE/../../oracle/stub" && pwd)
WORK=$(mktemp -d)
trap 'rm -rf "$WORK"' EXIT
M=$REF/preprocessing/mesh
S=$REF/preprocessing/spline
g++ -O2 -std=c++17 -I"$M/include" -I"$REF/include" -o "$WORK/tubular_mesh" "$M"/src/*.cpp
g++ -O2 -std=c++17 -fopenmp -I"$STUB" -I"$REF/include" -o "$WORK/spline" \
	"$S/BasicDataStructure.cpp" "$S/kernel.cpp" "$S/KnotInsertion.cpp" "$S/main.cpp" "$S/BSplineBasis.cpp"
g++ -O2 -std=c++17 -I"$STUB" -I"$REF/solvers/cpu/include" -I"$REF/include" \
	-o "$WORK/iga_pack" "$REF/solvers/cpu/src/iga_pack.cpp"
CASE=$WORK/case
mkdir -p "$CASE"
# A parent segment along +x splitting into two narrower daughters (SWC: id type x y z radius parent).
cat > "$CASE/skeleton_initial.swc" <<'SWC'
1 2 0.0 0.0 0.0 0.5 -1
2 2 2.0 0.0 0.0 0.5 1
3 2 4.0 1.2 0.0 0.4 2
4 2 4.0 -1.2 0.0 0.4 2
SWC
cat > "$CASE/simulation_config.json" <<'JSON'
{
  "schema_version": 4,
  "dimension": "3d",
  "geometry": {"kind": "swc_network", "file": "skeleton_initial.swc", "length_scale_to_m": 1.0},
  "mesh": {
    "cross_section": {"kind": "circle", "target_size": 0.25},
    "smoothing": {"iterations": 0, "bifurcation_ratio": 0.0, "noise_ratio": 0.0},
    "centerline": {"target_spacing": 1.0, "max_spacing_over_diameter": 1.0, "max_turn_degrees": 12.0,
      "max_diameter_change_fraction": 0.15, "maximum_curvature_radius_product": 0.8},
    "junction": {"max_spacing_over_diameter": 0.25, "upstream_clearance_over_diameter": 1.0,
      "downstream_clearance_over_diameter": 1.5, "minimum_angle_degrees": 10.0, "maximum_radius_ratio": 8.0,
      "optimization_iterations": 0},
    "quality": {"minimum_scaled_jacobian": 0.1, "check_self_intersection": true, "collision_safety_factor": 1.0}
  },
  "fields": [{"name": "velocity", "kind": "vector3"}, {"name": "pressure", "kind": "pressure"}],
  "time": {"dt": 0.1, "steps": 2},
  "equation_systems": [{"name": "blood_flow", "kind": "navier_stokes", "unknowns": ["velocity", "pressure"],
    "viscosity": 1.0, "density": 1.0, "time_integration": "backward_euler"}],
  "boundaries": [
    {"label": 0, "name": "wall", "conditions": [{"field": "velocity", "type": "dirichlet", "value": [0.0, 0.0, 0.0]}]},
    {"label": 1, "name": "inlet", "conditions": [{"field": "velocity", "type": "dirichlet",
      "profile": "initial_velocityfield.txt", "scale": 0.01}]},
    {"label": 2, "name": "outlet", "conditions": [{"field": "pressure", "type": "pressure_traction", "value": 0.0}]},
    {"label": 3, "name": "outlet2", "conditions": [{"field": "pressure", "type": "pressure_traction", "value": 0.0}]}
  ]
}
JSON
"$WORK/tubular_mesh" pipeline "$CASE" "$REF/Input" > "$WORK/mesh.log"
OMP_NUM_THREADS=2 "$WORK/spline" "$CASE/" --no-legacy-text > "$WORK/spline.log"
E=$(awk '/^CELLS/ {print $2}' "$CASE/controlmesh.vtk")
python3 -c "import sys; open(sys.argv[1],'w').write('0\n'*int(sys.argv[2]))" "$CASE/bzmeshinfo.txt.epart.1" "$E"
"$WORK/iga_pack" "$CASE" 1 "$CASE/bifurcation-1.ntiga" > "$WORK/pack.log"
OUT=$HERE/reference_bifurcation
mkdir -p "$OUT"
for f in bifurcation-1.ntiga controlmesh.vtk initial_velocityfield.txt simulation_config.json; do
	xz -9 -c "$CASE/$f" > "$OUT/$f.xz"
done
echo "wrote $OUT ($E elements)"
