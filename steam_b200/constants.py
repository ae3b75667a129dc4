"""Physical and model constants of the STEAM path (steam/constants.py:1-15)."""

specific_heat_dry_air = 1004.0          # cp [J/(kg K)]
latent_heat_vaporization = 2.5e6        # Lv [J/kg]
gravity = 9.81                          # g [m/s^2]
gas_constant_dry_air = 287.04           # Rd [J/(kg K)]

# Horizontal Hurst exponent and the Haar-to-Mexican-hat amplitude factor
# (lambda) calibrated together; they must change together.
hurst_horizontal = 0.45
haar_to_mhat = 0.25518

# Vertical anisotropy exponent H_z of k_z = l_s (k / l_s)^H_z.
hurst_vertical_anisotropy = 5 / 9
