"""Output contract: the Zarr v3 result store and status.json (solver/io/zarr_writer.py, status.py)."""
