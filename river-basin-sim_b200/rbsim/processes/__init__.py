"""Processes advanced at sync points or each step: point inflows and morphology."""
