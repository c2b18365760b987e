"""The polar CSV writer produces the reference's layout (Polar.cpp:126-164):
the same header lines and columns, empty separation fields where attached."""
import cfd_b200 as cb


def _result(status, cl, cd, upper, lower):
    r = cb.Result()
    r.status, r.iterations, r.continuity = status, 812, 3.25e-7
    r.lift_coefficient, r.drag_coefficient, r.moment_coefficient = cl, cd, -0.0123
    r.pressure_drag_coefficient, r.friction_drag_coefficient = 0.6 * cd, 0.4 * cd
    r.separation_upper_chord_fraction, r.separation_lower_chord_fraction = upper, lower
    return r


def test_header_and_rows():
    text = cb.polar_csv([_result(0, 0.5, 0.02, 0.7125, -1.0), _result(1, 1.1, 0.0, -1.0, -1.0)],
                        [4.0, 12.0], "NACA 2412", "Fine", 3e6, 50.0)
    lines = text.splitlines()
    assert lines[0] == "# cfd_simulator aerodynamic polar"
    assert lines[3] == "# reynolds,3e+06"
    assert lines[4] == "# freestream_speed_mps,50"
    assert lines[7] == "# continued_between_points,no"
    assert lines[10] == ("alpha_deg,cl,cd,cd_pressure,cd_friction,cm,l_over_d,"
                         "separation_upper_xc,separation_lower_xc,status,iterations,continuity_residual")
    assert lines[11] == ("4.000000,0.50000000,0.02000000,0.01200000,0.00800000,-0.01230000,"
                         "25.000000,0.712500,,converged,812,3.250000e-07")
    # Cd <= 0: l_over_d 0; attached both sides: empty separation fields
    assert lines[12].startswith("12.000000,1.10000000,0.00000000,")
    assert ",0.000000,,,iteration-limit,812," in lines[12]
