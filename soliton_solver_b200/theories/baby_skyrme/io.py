"""Output bundle of the theory (soliton_solver/theories/baby_skyrme/io.py): the same
file names and layout, formatted on the GPU by soliton_solver_b200.core.io."""
from __future__ import annotations

from soliton_solver_b200.core.io import output_data_bundle_core


def output_data_bundle(output_dir, h_Field, h_EnergyDensity, h_BaryonDensity, h_grid, xlen, ylen, number_coordinates=2,
                       number_total_fields=3, precision=32):
    arrays = {'grid': h_grid, 'Field': h_Field, 'EnergyDensity': h_EnergyDensity, 'BaryonDensity': h_BaryonDensity}
    bundle_spec = [('grid', 0, 'xGrid.dat'), ('grid', 1, 'yGrid.dat'), ('Field', 0, 'MagnetField1.dat'),
                   ('Field', 1, 'MagnetField2.dat'), ('Field', 2, 'MagnetField3.dat'),
                   ('BaryonDensity', 0, 'SkyrmionChargeDensity.dat'), ('EnergyDensity', 0, 'EnergyDensity.dat')]
    output_data_bundle_core(output_dir, h_Field=h_Field, h_grid=h_grid, xlen=xlen, ylen=ylen,
                            number_coordinates=number_coordinates, number_total_fields=number_total_fields,
                            precision=precision, bundle_spec=bundle_spec, arrays=arrays,
                            lattice_points_name="LatticePoints.dat", lattice_vectors_name="LatticeVectors.dat",
                            field_dump_name="Field.dat")
