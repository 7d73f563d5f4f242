"""gpx-pex: a B200-native quasi-static capacitance extractor (field-solver path)."""
